// Output of the quasi-dynamic driver at the reference's strides (see writer.hpp).
#include <cstdint>
#include <cstring>

#include "common.cuh"
#include "qd.hpp"
#include "writer.hpp"

namespace scy {

namespace {
constexpr int kSlots = 8;
constexpr int32_t kVecClassId = 1211214;

uint32_t be32(uint32_t v) { return __builtin_bswap32(v); }
uint64_t be64(uint64_t v) { return __builtin_bswap64(v); }

bool put_vec(FILE* f, const double* v, size_t n) {
  const int32_t hdr[2] = {(int32_t)be32((uint32_t)kVecClassId), (int32_t)be32((uint32_t)n)};
  if (fwrite(hdr, sizeof(hdr), 1, f) != 1) return false;
  std::vector<uint64_t> b(n);
  for (size_t i = 0; i < n; ++i) {
    uint64_t u;
    std::memcpy(&u, v + i, 8);
    b[i] = be64(u);
  }
  return fwrite(b.data(), 8, n, f) == n;
}
}  // namespace

OutputWriter::~OutputWriter() {
  {
    std::lock_guard<std::mutex> lk(mu);
    stop = true;
  }
  cv.notify_all();
  if (worker.joinable()) worker.join();
  for (auto& kv : files) fclose(kv.second);
  for (auto& s : slots) {
    if (s.h1) cudaFreeHost(s.h1);
    if (s.h2) cudaFreeHost(s.h2);
    if (s.ev) cudaEventDestroy(s.ev);
  }
}

int OutputWriter::open(const std::string& outputDir, int s1, int s2, double maxTime, int append_mode,
                       const QDContext& q) {
  if (q.pl) {
    set_error("the output writer covers the linear-elastic driver");
    return SCY_ERR_ARG;
  }
  dir = outputDir;
  stride1D = s1;
  stride2D = s2;
  max_time = maxTime;
  append = append_mode;
  Ny = q.Ny;
  Nz = q.Nz;
  N = q.N;
  n1 = 3 * (size_t)Ny + 10 * (size_t)Nz;
  n2 = stride2D > 0 ? 2 * (size_t)N : 0;
  slots.resize(kSlots);
  for (auto& s : slots) {
    SCY_CUDA_TRY(cudaMallocHost((void**)&s.h1, n1 * 8));
    if (n2) SCY_CUDA_TRY(cudaMallocHost((void**)&s.h2, n2 * 8));
    SCY_CUDA_TRY(cudaEventCreateWithFlags(&s.ev, cudaEventDisableTiming));
  }
  worker = std::thread([this] { run(); });
  return SCY_OK;
}

FILE* OutputWriter::file(const std::string& name, bool binary) {
  auto it = files.find(name);
  if (it != files.end()) return it->second;
  FILE* f = fopen((dir + name).c_str(), append ? (binary ? "ab" : "a") : (binary ? "wb" : "w"));
  if (f) files[name] = f;
  return f;
}

int OutputWriter::on_step(QDContext& q, long step, double t, double dt) {
  {
    std::lock_guard<std::mutex> lk(mu);
    if (io_error) {
      set_error("%s", io_msg.c_str());
      return SCY_ERR_IO;
    }
  }
  const bool do1 = stride1D > 0 && (t == max_time || step % stride1D == 0);
  const bool do2 = stride2D > 0 && (t == max_time || step % stride2D == 0);
  if (!do1 && !do2) return SCY_OK;
  Slot& s = slots[next];
  {
    std::unique_lock<std::mutex> lk(mu);
    cv.wait(lk, [&] { return !s.busy; });
  }
  cudaStream_t st = q.sbp.stream;
  const double* var = q.rk[V_VAR].as<double>();
  if (do1) {
    double* h = s.h1;
    SCY_CUDA_TRY(cudaMemcpy2DAsync(h, 8, q.u.p, (size_t)Nz * 8, 8, Ny, cudaMemcpyDeviceToHost, st));
    h += Ny;
    auto cp = [&](const void* src, size_t n) -> int {
      SCY_CUDA_TRY(cudaMemcpyAsync(h, src, n * 8, cudaMemcpyDeviceToHost, st));
      h += n;
      return SCY_OK;
    };
    SCY_TRY(cp(q.bcR.p, Nz));
    SCY_TRY(cp(q.bcT.p, Ny));
    SCY_TRY(cp(q.bcL.p, Nz));
    SCY_TRY(cp(q.bcB.p, Ny));
    SCY_TRY(cp(q.bcRShift.p, Nz));
    SCY_TRY(cp(var + q.fp.slip_off, Nz));
    SCY_TRY(cp(q.slipVel.p, Nz));
    SCY_TRY(cp(q.tauP.p, Nz));
    SCY_TRY(cp(q.tauQSP.p, Nz));
    SCY_TRY(cp(q.strength.p, Nz));
    SCY_TRY(cp(var + q.fp.psi_off, Nz));
    SCY_TRY(cp(q.fsN.p, Nz));
  }
  if (do2) {
    SCY_TRY(q.sbp.apply(SCY_OP_MUXDY, q.u.as<double>(), q.sxy.as<double>()));
    SCY_CUDA_TRY(cudaMemcpyAsync(s.h2, q.u.p, N * 8, cudaMemcpyDeviceToHost, st));
    SCY_CUDA_TRY(cudaMemcpyAsync(s.h2 + N, q.sxy.p, N * 8, cudaMemcpyDeviceToHost, st));
  }
  SCY_CUDA_TRY(cudaEventRecord(s.ev, st));
  {
    std::lock_guard<std::mutex> lk(mu);
    s.step = step;
    s.t = t;
    s.dt = dt;
    s.do1 = do1;
    s.do2 = do2;
    s.busy = 1;
    queue.push_back(next);
  }
  cv.notify_all();
  next = (next + 1) % kSlots;
  return SCY_OK;
}

void OutputWriter::write_slot(Slot& s) {
  bool ok = true;
  if (s.do1) {
    FILE* ft = file("med_time1D.txt", false);
    FILE* fd = file("med_dt1D.txt", false);
    ok = ok && ft && fd && fprintf(ft, "%.15e\n", s.t) > 0 && fprintf(fd, "%.15e\n", s.dt) > 0;
    const double* h = s.h1;
    const double* surf = h;
    const double* bcR = surf + Ny;
    const double* bcT = bcR + Nz;
    const double* bcL = bcT + Ny;
    const double* bcB = bcL + Nz;
    const double* shift = bcB + Ny;
    const double* f = shift + Nz;
    struct Rec {
      const char* name;
      const double* v;
      size_t n;
    };
    const Rec recs[] = {{"surfDisp", surf, (size_t)Ny},
                        {"momBal_bcR", bcR, (size_t)Nz},
                        {"momBal_bcT", bcT, (size_t)Ny},
                        {"momBal_bcL", bcL, (size_t)Nz},
                        {"momBal_bcB", bcB, (size_t)Ny},
                        {"momBal_bcRShift", records_bcRShift == 0 ? shift : bcR, (size_t)Nz},
                        {"slip", f, (size_t)Nz},
                        {"slipVel", f + Nz, (size_t)Nz},
                        {"tauP", f + 2 * Nz, (size_t)Nz},
                        {"tauQSP", f + 3 * Nz, (size_t)Nz},
                        {"strength", f + 4 * Nz, (size_t)Nz},
                        {"psi", f + 5 * Nz, (size_t)Nz},
                        {"sNEff", f + 6 * Nz, (size_t)Nz}};
    for (const Rec& r : recs) {
      FILE* fv = file(r.name, true);
      ok = ok && fv && put_vec(fv, r.v, r.n);
    }
    ++records_bcRShift;
    ++written1D;
  }
  if (s.do2) {
    FILE* ft = file("med_time2D.txt", false);
    FILE* fd = file("med_dt2D.txt", false);
    ok = ok && ft && fd && fprintf(ft, "%.15e\n", s.t) > 0 && fprintf(fd, "%.15e\n", s.dt) > 0;
    FILE* fu = file("momBal_u", true);
    FILE* fs = file("momBal_sxy", true);
    ok = ok && fu && fs && put_vec(fu, s.h2, N) && put_vec(fs, s.h2 + N, N);
    ++written2D;
  }
  if (!ok) {
    std::lock_guard<std::mutex> lk(mu);
    io_error = 1;
    io_msg = "writing output under '" + dir + "' failed";
  }
}

void OutputWriter::run() {
  for (;;) {
    int idx;
    {
      std::unique_lock<std::mutex> lk(mu);
      cv.wait(lk, [&] { return stop || !queue.empty(); });
      if (queue.empty()) return;  // stop requested and nothing left
      idx = queue.front();
    }
    Slot& s = slots[idx];
    if (cudaEventSynchronize(s.ev) != cudaSuccess) {
      std::lock_guard<std::mutex> lk(mu);
      io_error = 1;
      io_msg = "output copy failed";
    } else {
      write_slot(s);
    }
    {
      std::lock_guard<std::mutex> lk(mu);
      queue.pop_front();
      s.busy = 0;
    }
    cv.notify_all();
  }
}

int OutputWriter::flush() {
  {
    std::unique_lock<std::mutex> lk(mu);
    cv.wait(lk, [&] { return queue.empty(); });
  }
  for (auto& kv : files) fflush(kv.second);
  std::lock_guard<std::mutex> lk(mu);
  if (io_error) {
    set_error("%s", io_msg.c_str());
    return SCY_ERR_IO;
  }
  return SCY_OK;
}

}  // namespace scy
