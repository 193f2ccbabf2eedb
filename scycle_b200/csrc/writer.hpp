// Output of the quasi-dynamic driver at the reference's strides
// (StrikeSlip_LinearElastic_qd::timeMonitor, strikeSlip_linearElastic_qd.cpp:417-462):
//   every stride1D-th step (and at maxTime): med_time1D.txt / med_dt1D.txt
//   (writeStep1D :466-495, "%.15e\n"), LinearElastic::writeStep1D
//   (linearElastic.cpp:623-655: surfDisp, momBal_bcR, momBal_bcT, momBal_bcL,
//   momBal_bcB, momBal_bcRShift) and Fault::writeStep (fault.cpp:512-557:
//   slip, slipVel, tauP, tauQSP, strength, psi, sNEff);
//   every stride2D-th step: med_time2D.txt / med_dt2D.txt and
//   LinearElastic::writeStep2D (:659-686: momBal_u, momBal_sxy).
// Vec files are PETSc binary with one record appended per output step
// (big-endian int32 class id 1211214, int32 length, float64 values), which
// the reference's MATLAB readers load.  As in the reference, the records of
// momBal_bcRShift after the first hold bcR (linearElastic.cpp:649).
//
// The device fields of a step are copied into a ring of pinned buffers on
// the driver's stream; a worker thread waits for each copy and appends the
// records, so the integration does not wait for the file system.
#pragma once
#include <condition_variable>
#include <cstdio>
#include <deque>
#include <map>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include <cuda_runtime.h>

namespace scy {

struct QDContext;

struct OutputWriter {
  std::string dir;
  int stride1D = 0, stride2D = 0;
  double max_time = 0.0;
  int append = 0;  // 1: append to existing files (a restart), 0: start them anew
  ~OutputWriter();
  int open(const std::string& outputDir, int s1, int s2, double maxTime, int append_mode, const QDContext& q);
  // timeMonitor's output part for step `step` at time t with step size dt
  int on_step(QDContext& q, long step, double t, double dt);
  int flush();  // waits for every queued step to be written
  long written1D = 0, written2D = 0;

 private:
  struct Slot {
    double* h1 = nullptr;  // 1D payload (pinned)
    double* h2 = nullptr;  // 2D payload (pinned)
    cudaEvent_t ev = nullptr;
    long step = 0;
    double t = 0, dt = 0;
    int do1 = 0, do2 = 0, busy = 0;
  };
  int Ny = 0, Nz = 0;
  long N = 0;
  size_t n1 = 0, n2 = 0;
  std::vector<Slot> slots;
  int next = 0;
  std::map<std::string, FILE*> files;
  int records_bcRShift = 0;
  std::thread worker;
  std::mutex mu;
  std::condition_variable cv;
  std::deque<int> queue;
  bool stop = false;
  int io_error = 0;
  std::string io_msg;
  void run();
  void write_slot(Slot& s);
  FILE* file(const std::string& name, bool binary);
};

}  // namespace scy
