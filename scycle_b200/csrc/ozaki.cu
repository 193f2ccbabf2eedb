// FP64-accurate products on the integer tensor cores (see ozaki.hpp).
//
// ozk_gemm_kernel<S, T>: one CTA of 128 threads per output tile of 128 rows
// x CN columns.  Thread 0 of warp 0 streams 64-byte K slices of the S digit
// planes of both operands into a ring of shared-memory stages by TMA
// (cp.async.bulk.tensor, 64-byte swizzle, completion on an mbarrier per
// stage); thread 0 of warp 1 issues, per stage and per 32-byte K step, the
// S(S+1)/2 digit products (tcgen05.mma.cta_group::1.kind::i8, both operands
// K-major in shared memory, signed 8-bit, 32-bit integer accumulators) into
// S accumulators of 128 x CN in tensor memory, one per digit-weight group
// (the products of one X plane with a stack of W planes as one MMA of N up
// to 256, see ozk_issue_kstep), and frees each stage with tcgen05.commit on
// its "empty" mbarrier.  After
// the last stage all four warps read their 32 rows of the accumulators
// (tcgen05.ld 32x32b), combine the groups with their powers of two, apply
// the row and column exponents (loaded by warps 2 and 3 while the products
// run) and store their row segments.
//
// Two digit formats: signed 8-bit digits multiplied by tcgen05.mma
// kind::i8 into 32-bit integer accumulators, or the same digits held in
// bf16 (every integer of magnitude <= 256 is exact there) multiplied by
// kind::f16 into FP32 accumulators, exact while every partial sum stays
// below 2^24 in magnitude (S * 64 * 64 * Kp < 2^24, checked on the host).
// The products are bit-identical; which is faster depends on the tensor
// pipe's integer and bf16 rates, so callers time both.
//
// Three shapes: one CTA per SM per tile (all 512 tensor-memory columns, CN
// = 144 / 112 / 96 / 64 columns for S = 3 / 4 / 5 / 6-7, up to four
// stages); for S <= 5, two CTAs per SM (256 columns each, CN = 64 / 64 / 48,
// two stages), where one CTA's epilogue overlaps the other's products; and
// for S <= 5 the persistent ozk_gemm_pers_kernel (one CTA per SM walking the
// tiles of width 64 / 64 / 48 with two accumulator sets).
//
// Every mbarrier wait is bounded (2^20 polls).  A wait that runs out marks
// the tile's rows in the caller's status words; the producer then waits
// (bounded) for the copies it issued that nobody consumed, the epilogue
// waits (bounded) for the issued products, and tensor memory is freed
// before the CTA exits.  TMA loads read this GPU's own memory only and use
// no cluster multicast.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "ozaki.hpp"
#include "tma.cuh"

namespace scy {
namespace {

constexpr int OZK_BM = 128;  // rows per tile (tensor-memory lanes)
constexpr int OZK_BK = 64;   // bytes of K per stage (one 64-byte swizzle row)
constexpr int OZK_POLLS = 1 << 20;
constexpr int OZK_SMEM_BUDGET = 220 * 1024;

// PAIR = 0: one CTA per SM; PAIR = 1: two (S <= 5)
__host__ __device__ constexpr int ozk_cn(int S, int pair = 0) {
  return pair ? (S <= 4 ? 64 : 48) : (S <= 3 ? 144 : S == 4 ? 112 : S == 5 ? 96 : 64);
}
__host__ __device__ constexpr int ozk_tmem_cols(int pair) { return pair ? 256 : 512; }
__host__ __device__ constexpr int ozk_stage_bytes(int S, int pair = 0) {
  return S * OZK_BM * OZK_BK + S * ozk_cn(S, pair) * OZK_BK;
}
__host__ __device__ constexpr int ozk_stages(int S, int pair = 0) {
  return pair ? 2 : OZK_SMEM_BUDGET / ozk_stage_bytes(S) > 4 ? 4 : OZK_SMEM_BUDGET / ozk_stage_bytes(S);
}
// the stage ring starts on a 1024-byte (one CTA per SM) or 512-byte (two)
// boundary: the 64-byte swizzle repeats every 512 bytes
__host__ __device__ constexpr int ozk_align(int pair) { return pair ? 512 : 1024; }
__host__ __device__ constexpr int ozk_smem_bytes(int S, int pair = 0) {
  return ozk_stages(S, pair) * ozk_stage_bytes(S, pair) + ozk_align(pair);
}
// the persistent shape (S <= 5): the two-CTAs-per-SM tile width (S * CN <=
// 256, so two accumulator sets fit the 512 tensor-memory columns) and as
// many stages of that width as fit one CTA's shared memory (at most four)
__host__ __device__ constexpr int ozk_pers_stages(int S) {
  return (227 * 1024 - 2048) / ozk_stage_bytes(S, 1) > 4 ? 4 : (227 * 1024 - 2048) / ozk_stage_bytes(S, 1);
}
__host__ __device__ constexpr int ozk_pers_smem_bytes(int S) { return ozk_pers_stages(S) * ozk_stage_bytes(S, 1) + 1024; }
// per CTA beside the stages: the reserved kilobyte, the barriers and the
// epilogue's exponent factors (CN + 128 doubles)
static_assert(2 * (ozk_smem_bytes(5, 1) + 1024 + 256 + 8 * (ozk_cn(5, 1) + 128)) <= 228 * 1024,
              "two CTAs per SM do not fit");
static_assert(2 * (ozk_smem_bytes(4, 1) + 1024 + 256 + 8 * (ozk_cn(4, 1) + 128)) <= 228 * 1024,
              "two CTAs per SM do not fit");
static_assert(2 * (ozk_smem_bytes(3, 1) + 1024 + 256 + 8 * (ozk_cn(3, 1) + 128)) <= 228 * 1024,
              "two CTAs per SM do not fit");

// shared-memory matrix descriptor (tcgen05 format): K-major operand whose
// rows are 64 bytes with 64-byte swizzling, 8-row groups 512 bytes apart
__device__ __forceinline__ uint64_t umma_desc_sw64(uint32_t saddr) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3FFFu);  // start address, 16-byte units
  d |= (uint64_t)1u << 16;                  // leading byte offset (unused by swizzled K-major layouts)
  d |= (uint64_t)(512u >> 4) << 32;         // stride byte offset: next 8-row group
  d |= (uint64_t)1u << 46;                  // descriptor version of sm_100
  d |= (uint64_t)4u << 61;                  // layout: 64-byte swizzle
  return d;
}

// 2^e as a double (exact), by its bit pattern in the normal range
__device__ __forceinline__ double pow2i(int e) {
  return (e >= -1022 && e <= 1023) ? __longlong_as_double((long long)(e + 1023) << 52) : ldexp(1.0, e);
}

// instruction descriptor: signed 8-bit A and B, K-major, 32-bit integer
// accumulator, M = 128, N = n
__host__ __device__ constexpr uint32_t umma_idesc_s8(int n) {
  return (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(OZK_BM >> 4) << 24);
}

// instruction descriptor: bf16 A and B, K-major, FP32 accumulator, M = 128,
// N = n
__host__ __device__ constexpr uint32_t umma_idesc_bf16(int n) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(OZK_BM >> 4) << 24);
}

__device__ __forceinline__ void umma_s8(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                        uint32_t accumulate) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
      " tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem_d),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
      : "memory");
}

__device__ __forceinline__ void umma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                          uint32_t accumulate) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
      " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem_d),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
      : "memory");
}

__device__ __forceinline__ void umma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&v)[16]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15}, [%16];"
      : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]), "=r"(v[8]),
        "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
      : "r"(taddr));
}

// The digit products of one 32-byte K step: X plane p times the stack of W
// planes 1 .. S+1-p.  Their products belong to the consecutive groups
// p-1 .. S-1, whose accumulators are consecutive in tensor memory, and the
// W planes are consecutive CN-row blocks of the stage, so one MMA of N =
// planes x CN (at most 256) covers as many of them as fit: the A tile is read
// once per MMA instead of once per product.  Integer (and the exact FP32)
// sums are the same in any order.  first: the tile's first K step (the
// products of X plane 1 start every group).
template <int S, int CN, int BF>
__device__ __forceinline__ void ozk_issue_kstep(uint32_t tacc, uint32_t xa, uint32_t wa, int ks, bool first) {
  constexpr int PER = 256 / CN;  // W planes per MMA
#pragma unroll
  for (int p = 1; p <= S; ++p) {
#pragma unroll
    for (int j0 = 1; j0 <= S + 1 - p; j0 += PER) {
      const int np = (S + 2 - p - j0) < PER ? (S + 2 - p - j0) : PER;
      const uint64_t ad = umma_desc_sw64(xa + (p - 1) * OZK_BM * OZK_BK + ks * 32);
      const uint64_t bd = umma_desc_sw64(wa + (j0 - 1) * CN * OZK_BK + ks * 32);
      const uint32_t idesc = BF ? umma_idesc_bf16(np * CN) : umma_idesc_s8(np * CN);
      const uint32_t acc = (first && p == 1) ? 0u : 1u;
      if (BF)
        umma_bf16(tacc + (p + j0 - 2) * CN, ad, bd, idesc, acc);
      else
        umma_s8(tacc + (p + j0 - 2) * CN, ad, bd, idesc, acc);
    }
  }
}

template <int S, typename T, int PAIR, int BF>
__global__ void __launch_bounds__(128, PAIR ? 2 : 1)
    ozk_gemm_kernel(const __grid_constant__ CUtensorMap mx, const __grid_constant__ CUtensorMap mw,
                    const int* __restrict__ ex, const int* __restrict__ ew, T* __restrict__ D, long ldd, int rows,
                    int cout, int nks, unsigned* __restrict__ status, int rows_per_status, unsigned bit) {
  constexpr int CN = ozk_cn(S, PAIR);
  constexpr int XB = S * OZK_BM * OZK_BK;
  constexpr int WB = S * CN * OZK_BK;
  constexpr int ST = ozk_stages(S, PAIR);
  constexpr int TC = ozk_tmem_cols(PAIR);
  constexpr unsigned AL = ozk_align(PAIR);
  static_assert(S * CN <= TC, "accumulators exceed tensor memory");
  static_assert(!PAIR || S <= 5, "two CTAs per SM only for S <= 5");
  static_assert(CN % 16 == 0 && CN >= 16 && CN <= 256, "invalid MMA N");
  extern __shared__ __align__(1024) unsigned char ozk_smem_raw[];
  __shared__ __align__(8) uint64_t full[ST], empty[ST], done;
  __shared__ uint32_t tmem_slot;
  __shared__ int consumed, failed;
  __shared__ double s_sw[CN], s_xs[OZK_BM];  // 2^ew of the tile's columns, 2^ex of its rows
  // tiles on a 1024- or 512-byte boundary (the swizzle pattern repeats every 512 B)
  unsigned char* smem = ozk_smem_raw + ((AL - (smem_u32(ozk_smem_raw) & (AL - 1))) & (AL - 1));
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  // column tiles vary fastest (the CTAs that run together share a row tile
  // of X and spread over the tiles of W), and each CTA starts its K loop at
  // its own stage (integer partial sums are exact in any order), so the
  // CTAs reading one W tile at a time read different parts of it
  const int c0 = blockIdx.x * CN, m0 = blockIdx.y * OZK_BM;

  if (threadIdx.x == 0) {
    for (int i = 0; i < ST; ++i) {
      mbar_init(&full[i], 1);
      mbar_init(&empty[i], 1);
    }
    mbar_init(&done, 1);
    fence_mbar_init();
    consumed = 0;
    failed = 0;
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_slot)),
                 "n"(TC)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = tmem_slot;

  // K in 32-byte MMA steps (nks), two per 64-byte stage; the last stage may
  // hold one.  N of the products: the tile's columns rounded up to 16 (the
  // last column tile is narrower than CN)
  const int nkb = (nks + 1) / 2;
  const int rot = (int)((blockIdx.x * 7u + blockIdx.y) % (unsigned)nkb);
  const int nmma = max(32, min(CN, (cout - c0 + 15) / 16 * 16));
  int issued = 0;
  if (warp >= 2) {
    // the epilogue's exponent factors, loaded while the products run
    for (int i = threadIdx.x - 64; i < CN + OZK_BM; i += 64) {
      if (i < CN)
        s_sw[i] = c0 + i < cout ? pow2i(ew[c0 + i]) : 0.0;
      else
        s_xs[i - CN] = m0 + (i - CN) < rows ? pow2i(ex[m0 + (i - CN)]) : 0.0;
    }
  }
  if (warp == 0 && lane == 0) {
    // producer
    for (int q = 0; q < nkb; ++q) {
      const int st = q % ST, kb = (q + rot) % nkb;
      if (q >= ST && !mbar_wait(&empty[st], ((q / ST) - 1) & 1, OZK_POLLS)) {
        failed = 1;
        break;
      }
      unsigned char* sx = smem + st * (XB + WB);
      mbar_expect_tx(&full[st], XB + WB);
      // x coordinate in digits: 64 bytes of K per stage
      tma_load_3d(sx, &mx, &full[st], kb * (OZK_BK / (BF ? 2 : 1)), m0, 0);
      tma_load_3d(sx + XB, &mw, &full[st], kb * (OZK_BK / (BF ? 2 : 1)), c0, 0);
      ++issued;
    }
  } else if (warp == 1 && lane == 0) {
    // MMA issuer
    int q = 0;
    for (; q < nkb; ++q) {
      const int st = q % ST, kb = (q + rot) % nkb;
      if (!mbar_wait(&full[st], (q / ST) & 1, OZK_POLLS)) {
        failed = 1;
        break;
      }
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const uint32_t xa = smem_u32(smem + st * (XB + WB));
      const uint32_t wa = xa + XB;
#pragma unroll
      for (int ks = 0; ks < 2; ++ks) {
        if (2 * kb + ks >= nks) break;
        ozk_issue_kstep<S, CN, BF>(tmem, xa, wa, ks, q == 0 && ks == 0);
      }
      umma_commit(&empty[st]);
    }
    consumed = q;
    umma_commit(&done);  // arrives once every product issued above has completed
  }
  __syncthreads();
  if (warp == 0 && lane == 0) {
    // copies issued but never consumed (only after a wait ran out)
    for (int q = consumed; q < issued; ++q) mbar_wait(&full[q % ST], (q / ST) & 1, OZK_POLLS);
  }
  // one decision for the whole block: the warp-collective tensor-memory
  // loads below run in every warp or in none
  const bool ok = __syncthreads_and(mbar_wait(&done, 0, OZK_POLLS) ? 1 : 0) && !failed;
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  if (!ok) {
    if (threadIdx.x == 0 && status) {
      const int r1 = min(m0 + OZK_BM, rows) - 1;
      for (int q = m0 / rows_per_status; q <= r1 / rows_per_status; ++q) atomicOr(status + q, bit);
    }
  } else {
    // epilogue: warp w owns tensor-memory lanes 32 w .. 32 w + 31 (rows);
    // a thread combines its row's groups, 16 columns at a time, applies the
    // exponent factors (exact powers of two, loaded during the products)
    // and stores the 16 values of its row segment
    const int rl = warp * 32 + lane, row = m0 + rl;
    const double xs = s_xs[rl];
    const uint32_t tl = tmem + ((uint32_t)(warp * 32) << 16);
#pragma unroll 1
    for (int cc = 0; cc < nmma; cc += 16) {
      uint32_t v[S][16];
#pragma unroll
      for (int g = 0; g < S; ++g) tmem_ld16(tl + g * CN + cc, v[g]);
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
      double acc[16];
      if constexpr (S <= 5) {
        // sum_g P_g 2^(-7 (g+2)) as one 64-bit integer (|P_g| < 2^24, so
        // the Horner sum stays below 2^52) times 2^(-7 (S+1)): exact, the
        // same value as the FP64 sum below, with one conversion per output
#pragma unroll
        for (int q = 0; q < 16; ++q) {
          long long h = 0;
#pragma unroll
          for (int g = 0; g < S; ++g) h = (h << 7) + (long long)(BF ? (int)__uint_as_float(v[g][q]) : (int)v[g][q]);
          acc[q] = (double)h * pow2i(-7 * (S + 1));
        }
      } else {
#pragma unroll
        for (int q = 0; q < 16; ++q) acc[q] = 0.0;
#pragma unroll
        for (int g = S - 1; g >= 0; --g) {
          // smallest weights first
          const double wgt = pow2i(-7 * (g + 2));
#pragma unroll
          for (int q = 0; q < 16; ++q)
            acc[q] += (BF ? (double)__uint_as_float(v[g][q]) : (double)(int)v[g][q]) * wgt;
        }
      }
      if (row < rows) {
        T* drow = D + (long)row * ldd + c0 + cc;
#pragma unroll
        for (int q = 0; q < 16; ++q)
          if (c0 + cc + q < cout) drow[q] = (T)((acc[q] * xs) * s_sw[cc + q]);
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 1) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "n"(TC) : "memory");
}

// ozk_gemm_pers_kernel<S, T, BF> (S <= 5): the same product as a persistent
// kernel.  One CTA of 256 threads per SM walks the output tiles of 128 rows
// x CN columns (CN of the two-CTAs-per-SM shape, S * CN <= 256), tile t =
// blockIdx.x + k * gridDim.x (column tiles fastest), with the accumulators
// double-buffered in tensor memory (columns 0..255 for even, 256..511 for odd
// tiles of the CTA), so the epilogue of one tile runs while the products of
// the next are issued.  Thread 0 of warp 0 streams the K slices of all the
// CTA's tiles through one stage ring; thread 0 of warp 1 issues the products
// and marks a buffer's accumulators complete (accf, by tcgen05.commit);
// warps 4..7 (tensor-memory lanes 32 (w - 4) ..) read, combine and store
// them and mark the buffer free (acce, one arrival per warp).  Same digit
// formats and the same results as ozk_gemm_kernel.  Every wait is bounded;
// a role whose wait runs out stops, the others stop at their next bounded
// wait or at the shared flag, issued copies and products are awaited
// (bounded) before the tensor memory is freed, and the rows of every tile
// of the CTA are marked in the caller's status words.
template <int S, typename T, int BF>
__global__ void __launch_bounds__(256, 1)
    ozk_gemm_pers_kernel(const __grid_constant__ CUtensorMap mx, const __grid_constant__ CUtensorMap mw,
                         const int* __restrict__ ex, const int* __restrict__ ew, T* __restrict__ D, long ldd,
                         int rows, int cout, int nks, unsigned* __restrict__ status, int rows_per_status,
                         unsigned bit) {
  constexpr int CN = ozk_cn(S, 1);
  constexpr int XB = S * OZK_BM * OZK_BK;
  constexpr int WB = S * CN * OZK_BK;
  constexpr int ST = ozk_pers_stages(S);
  static_assert(S <= 5 && S * CN <= 256, "two accumulator sets must fit the tensor memory");
  static_assert(CN % 16 == 0 && CN >= 32, "invalid MMA N");
  extern __shared__ __align__(1024) unsigned char ozk_smem_raw[];
  __shared__ __align__(8) uint64_t full[ST], empty[ST], accf[2], acce[2], done;
  __shared__ uint32_t tmem_slot;
  __shared__ volatile int failed;
  __shared__ int issued_q, consumed_q;
  unsigned char* smem = ozk_smem_raw + ((1024u - (smem_u32(ozk_smem_raw) & 1023u)) & 1023u);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int ntc = (cout + CN - 1) / CN, ntr = (rows + OZK_BM - 1) / OZK_BM, ntiles = ntc * ntr;
  const int nkb = (nks + 1) / 2;

  if (threadIdx.x == 0) {
    for (int i = 0; i < ST; ++i) {
      mbar_init(&full[i], 1);
      mbar_init(&empty[i], 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(&accf[b], 1);
      mbar_init(&acce[b], 4);
    }
    mbar_init(&done, 1);
    fence_mbar_init();
    failed = 0;
    issued_q = 0;
    consumed_q = 0;
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 512;" ::"r"(smem_u32(&tmem_slot))
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = tmem_slot;

  if (warp == 0 && lane == 0) {
    // producer
    int q = 0;
    for (int t = blockIdx.x; t < ntiles && !failed; t += gridDim.x) {
      const int ct = t % ntc, rt = t / ntc, c0 = ct * CN, m0 = rt * OZK_BM;
      const int rot = (int)((ct * 7u + rt) % (unsigned)nkb);
      bool ok = true;
      for (int k = 0; k < nkb; ++k) {
        const int st = q % ST, kb = (k + rot) % nkb;
        if (q >= ST && !mbar_wait(&empty[st], ((q / ST) - 1) & 1, OZK_POLLS)) {
          failed = 1;
          ok = false;
          break;
        }
        unsigned char* sx = smem + st * (XB + WB);
        mbar_expect_tx(&full[st], XB + WB);
        tma_load_3d(sx, &mx, &full[st], kb * (OZK_BK / (BF ? 2 : 1)), m0, 0);
        tma_load_3d(sx + XB, &mw, &full[st], kb * (OZK_BK / (BF ? 2 : 1)), c0, 0);
        ++q;
      }
      if (!ok) break;
    }
    issued_q = q;
  } else if (warp == 1 && lane == 0) {
    // MMA issuer
    int q = 0, i = 0;
    for (int t = blockIdx.x; t < ntiles && !failed; t += gridDim.x, ++i) {
      const int ct = t % ntc, rt = t / ntc;
      const int rot = (int)((ct * 7u + rt) % (unsigned)nkb);
      const int b = i & 1;
      if (i >= 2 && !mbar_wait(&acce[b], ((i >> 1) - 1) & 1, OZK_POLLS)) {
        failed = 1;
        break;
      }
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const uint32_t tb = tmem + (uint32_t)(b * 256);
      bool ok = true;
      for (int k = 0; k < nkb; ++k) {
        const int st = q % ST, kb = (k + rot) % nkb;
        if (!mbar_wait(&full[st], (q / ST) & 1, OZK_POLLS)) {
          failed = 1;
          ok = false;
          break;
        }
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const uint32_t xa = smem_u32(smem + st * (XB + WB));
        const uint32_t wa = xa + XB;
#pragma unroll
        for (int ks = 0; ks < 2; ++ks) {
          if (2 * kb + ks >= nks) break;
          ozk_issue_kstep<S, CN, BF>(tb, xa, wa, ks, k == 0 && ks == 0);
        }
        umma_commit(&empty[st]);
        ++q;
      }
      if (!ok) break;
      umma_commit(&accf[b]);  // arrives once the tile's products have completed
    }
    consumed_q = q;
    umma_commit(&done);
  } else if (warp >= 4) {
    // epilogue
    const int wq = warp - 4;
    int i = 0;
    for (int t = blockIdx.x; t < ntiles; t += gridDim.x, ++i) {
      const int ct = t % ntc, rt = t / ntc, c0 = ct * CN, m0 = rt * OZK_BM;
      const int nmma = max(32, min(CN, (cout - c0 + 15) / 16 * 16));
      const int b = i & 1;
      const int row = m0 + wq * 32 + lane;
      const double xs = row < rows ? pow2i(ex[row]) : 0.0;
      const bool got = mbar_wait(&accf[b], (i >> 1) & 1, OZK_POLLS);
      if (!__all_sync(0xffffffffu, got ? 1 : 0) || failed) {
        failed = 1;
        break;
      }
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const uint32_t tl = tmem + ((uint32_t)(wq * 32) << 16) + (uint32_t)(b * 256);
#pragma unroll 1
      for (int cc = 0; cc < nmma; cc += 16) {
        uint32_t v[S][16];
#pragma unroll
        for (int g = 0; g < S; ++g) tmem_ld16(tl + g * CN + cc, v[g]);
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
        if (row < rows) {
          T* drow = D + (long)row * ldd + c0 + cc;
#pragma unroll
          for (int q2 = 0; q2 < 16; ++q2) {
            // the digit groups as one 64-bit integer (see ozk_gemm_kernel)
            long long h = 0;
#pragma unroll
            for (int g = 0; g < S; ++g)
              h = (h << 7) + (long long)(BF ? (int)__uint_as_float(v[g][q2]) : (int)v[g][q2]);
            const int c = c0 + cc + q2;
            if (c < cout) drow[q2] = (T)((((double)h * pow2i(-7 * (S + 1))) * xs) * pow2i(ew[c]));
          }
        }
      }
      asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
      __syncwarp();
      if (lane == 0) mbar_expect_tx(&acce[b], 0);  // this warp's arrival: the buffer's lanes are read
    }
  }
  __syncthreads();
  if (warp == 0 && lane == 0) {
    // copies issued but never consumed (only after a wait ran out)
    for (int q = consumed_q; q < issued_q; ++q) mbar_wait(&full[q % ST], (q / ST) & 1, OZK_POLLS);
  }
  const bool okd = __syncthreads_and(mbar_wait(&done, 0, OZK_POLLS) ? 1 : 0) && !failed;
  if (!okd && threadIdx.x == 0 && status) {
    for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
      const int m0 = (t / ntc) * OZK_BM, r1 = min(m0 + OZK_BM, rows) - 1;
      for (int qq = m0 / rows_per_status; qq <= r1 / rows_per_status; ++qq) atomicOr(status + qq, bit);
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 1) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 512;" ::"r"(tmem) : "memory");
}

// digits of one row per warp, in two coalesced passes over the row (the
// second from L1).  The first pass (lane l reads positions 32 t + l) gives
// the row maximum (a warp reduction) and so the row's exponent; in the
// second lane l takes the four consecutive positions 128 t + 4 l .. + 3 and
// writes their S digits with one store per plane (four bytes, or the four
// bf16 patterns of the digits: the upper halves of their FP32 patterns,
// exact for |d| <= 256).  Kp is a multiple of 4, so every store is aligned
// and inside the row.
template <typename Tin, int BF>
__global__ void __launch_bounds__(256) ozk_split_kernel(const Tin* __restrict__ X, long ldx, int rows, int K, int Kp,
                                                        int S, unsigned char* __restrict__ dig, long plane,
                                                        int* __restrict__ expo) {
  const int row = (int)((blockIdx.x * (long)blockDim.x + threadIdx.x) >> 5);
  const int lane = threadIdx.x & 31;
  if (row >= rows) return;
  const Tin* x = X + (long)row * ldx;
  double m = 0.0;
  for (int k = lane; k < K; k += 32) m = fmax(m, fabs((double)x[k]));
  m = warp_max(m);
  const int e = m > 0.0 ? ilogb(m) + 2 : 0;
  if (lane == 0) expo[row] = e;
  for (int k0 = 4 * lane; k0 < Kp; k0 += 128) {
    double t[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) t[u] = k0 + u < K ? ldexp((double)x[k0 + u], 7 - e) : 0.0;
    const long at = (long)row * Kp + k0;
    for (int i = 0; i < S; ++i) {
      uint32_t w0 = 0, w1 = 0;
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const double d = rint(t[u]);
        t[u] = (t[u] - d) * 128.0;
        if (BF) {
          const uint32_t h = __float_as_uint((float)d) >> 16;
          if (u < 2)
            w0 |= h << (16 * u);
          else
            w1 |= h << (16 * (u - 2));
        } else {
          w0 |= (uint32_t)(uint8_t)(int8_t)(int)d << (8 * u);
        }
      }
      if (BF)
        *reinterpret_cast<uint2*>(reinterpret_cast<uint16_t*>(dig) + (long)i * plane + at) = make_uint2(w0, w1);
      else
        *reinterpret_cast<uint32_t*>(dig + (long)i * plane + at) = w0;
    }
  }
}

// The same digits with the row held in registers (Kp <= 128 NC): lane l
// loads positions 128 c + 4 l .. + 3 once, takes the row maximum from them
// and writes the digits from them (one pass over the row in memory).
template <typename Tin, int BF, int NC>
__global__ void __launch_bounds__(256) ozk_split_reg_kernel(const Tin* __restrict__ X, long ldx, int rows, int K,
                                                            int Kp, int S, unsigned char* __restrict__ dig,
                                                            long plane, int* __restrict__ expo) {
  const int row = (int)((blockIdx.x * (long)blockDim.x + threadIdx.x) >> 5);
  const int lane = threadIdx.x & 31;
  if (row >= rows) return;
  const Tin* x = X + (long)row * ldx;
  double t[NC][4];
  double m = 0.0;
#pragma unroll
  for (int c = 0; c < NC; ++c)
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int k = 128 * c + 4 * lane + u;
      t[c][u] = k < K ? (double)x[k] : 0.0;
      m = fmax(m, fabs(t[c][u]));
    }
  m = warp_max(m);
  const int e = m > 0.0 ? ilogb(m) + 2 : 0;
  if (lane == 0) expo[row] = e;
#pragma unroll
  for (int c = 0; c < NC; ++c) {
    const int k0 = 128 * c + 4 * lane;
    if (k0 >= Kp) break;
#pragma unroll
    for (int u = 0; u < 4; ++u) t[c][u] = ldexp(t[c][u], 7 - e);
    const long at = (long)row * Kp + k0;
    for (int i = 0; i < S; ++i) {
      uint32_t w0 = 0, w1 = 0;
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const double d = rint(t[c][u]);
        t[c][u] = (t[c][u] - d) * 128.0;
        if (BF) {
          const uint32_t h = __float_as_uint((float)d) >> 16;
          if (u < 2)
            w0 |= h << (16 * u);
          else
            w1 |= h << (16 * (u - 2));
        } else {
          w0 |= (uint32_t)(uint8_t)(int8_t)(int)d << (8 * u);
        }
      }
      if (BF)
        *reinterpret_cast<uint2*>(reinterpret_cast<uint16_t*>(dig) + (long)i * plane + at) = make_uint2(w0, w1);
      else
        *reinterpret_cast<uint32_t*>(dig + (long)i * plane + at) = w0;
    }
  }
}

template <int S, typename T, int PAIR, int BF>
int prepare_one() {
  // the shared-memory limit is a per-device function attribute
  static unsigned long long attr_set = 0;
  int dev = 0;
  SCY_CUDA_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64 || !(attr_set >> dev & 1ull)) {
    SCY_CUDA_TRY(cudaFuncSetAttribute(ozk_gemm_kernel<S, T, PAIR, BF>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      ozk_smem_bytes(S, PAIR)));
    if (dev >= 0 && dev < 64) attr_set |= 1ull << dev;
  }
  return SCY_OK;
}

template <int S, typename T, int BF>
int prepare_pers() {
  static unsigned long long attr_set = 0;
  int dev = 0;
  SCY_CUDA_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64 || !(attr_set >> dev & 1ull)) {
    SCY_CUDA_TRY(cudaFuncSetAttribute(ozk_gemm_pers_kernel<S, T, BF>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      ozk_pers_smem_bytes(S)));
    if (dev >= 0 && dev < 64) attr_set |= 1ull << dev;
  }
  return SCY_OK;
}

template <int S, int BF>
int prepare_sb() {
  int rc = prepare_one<S, double, 0, BF>();
  if (rc == SCY_OK) rc = prepare_one<S, float, 0, BF>();
  if constexpr (S <= 5) {
    if (rc == SCY_OK) rc = prepare_one<S, double, 1, BF>();
    if (rc == SCY_OK) rc = prepare_one<S, float, 1, BF>();
    if (rc == SCY_OK) rc = prepare_pers<S, double, BF>();
    if (rc == SCY_OK) rc = prepare_pers<S, float, BF>();
  }
  return rc;
}

// multiprocessors of the current device (cached per device)
int sm_count() {
  static int cached[64] = {0};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return kNumSMs;
  if (!cached[dev]) {
    int n = 0;
    if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n < 1) n = kNumSMs;
    cached[dev] = n;
  }
  return cached[dev];
}

template <int S>
int prepare_s() {
  const int rc = prepare_sb<S, 0>();
  return rc != SCY_OK ? rc : prepare_sb<S, 1>();
}

template <int S, typename T, int PAIR, int BF>
int launch_gemm(const OzkOperand& x, const CUtensorMap& wmap, const OzkOperand& w, T* D, long ldd, int cout,
                cudaStream_t s, unsigned* status, int rows_per_status, unsigned bit) {
  constexpr int CN = ozk_cn(S, PAIR);
  {
    const int rc = prepare_one<S, T, PAIR, BF>();
    if (rc != SCY_OK) return rc;
  }
  const dim3 grid((cout + CN - 1) / CN, (x.rows + OZK_BM - 1) / OZK_BM);
  ozk_gemm_kernel<S, T, PAIR, BF><<<grid, 128, ozk_smem_bytes(S, PAIR), s>>>(
      x.map, wmap, x.expo.as<int>(), w.expo.as<int>(), D, ldd, x.rows, cout, x.Kp * x.esz / 32, status,
      rows_per_status, bit);
  SCY_LAUNCH_CHECK();
  return SCY_OK;
}

// the persistent shape: one CTA per SM (at most one per tile)
template <int S, typename T, int BF>
int launch_pers(const OzkOperand& x, const OzkOperand& w, T* D, long ldd, int cout, cudaStream_t s,
                unsigned* status, int rows_per_status, unsigned bit) {
  constexpr int CN = ozk_cn(S, 1);
  SCY_TRY((prepare_pers<S, T, BF>()));
  const long ntiles = (long)((cout + CN - 1) / CN) * ((x.rows + OZK_BM - 1) / OZK_BM);
  const int grid = (int)std::min<long>(ntiles, sm_count());
  ozk_gemm_pers_kernel<S, T, BF><<<grid, 256, ozk_pers_smem_bytes(S), s>>>(
      x.map, w.map_pair, x.expo.as<int>(), w.expo.as<int>(), D, ldd, x.rows, cout, x.Kp * x.esz / 32, status,
      rows_per_status, bit);
  SCY_LAUNCH_CHECK();
  return SCY_OK;
}

template <int S, typename T, int BF>
int launch_variant_b(const OzkOperand& x, const OzkOperand& w, T* D, long ldd, int cout, cudaStream_t s,
                     unsigned* status, int rps, unsigned bit, int pair) {
  if constexpr (S <= 5) {
    if (pair == 2) return launch_pers<S, T, BF>(x, w, D, ldd, cout, s, status, rps, bit);
    if (pair) return launch_gemm<S, T, 1, BF>(x, w.map_pair, w, D, ldd, cout, s, status, rps, bit);
  }
  return launch_gemm<S, T, 0, BF>(x, w.map, w, D, ldd, cout, s, status, rps, bit);
}

template <int S, typename T>
int launch_variant(const OzkOperand& x, const OzkOperand& w, T* D, long ldd, int cout, cudaStream_t s,
                   unsigned* status, int rps, unsigned bit, int pair) {
  if (x.esz == 2) return launch_variant_b<S, T, 1>(x, w, D, ldd, cout, s, status, rps, bit, pair);
  return launch_variant_b<S, T, 0>(x, w, D, ldd, cout, s, status, rps, bit, pair);
}

template <typename T>
int gemm_any(const OzkOperand& x, const OzkOperand& w, T* D, long ldd, int cout, cudaStream_t s, unsigned* status,
             int rps, unsigned bit, int pair) {
  pair = pair == 2 ? 2 : pair ? 1 : 0;
  if (x.S != w.S || x.Kp != w.Kp || x.K != w.K || x.esz != w.esz || cout > w.rows || cout < 1 || x.rows < 1 ||
      w.box_rows != ozk_cn(w.S) || x.box_rows != OZK_BM || rps < 1 ||
      (pair && (w.S > 5 || w.box_rows_pair != ozk_cn(w.S, 1)))) {
    set_error("ozk_gemm: operands do not match (S %d/%d, K %d/%d, cout %d, W rows %d, shape %d)", x.S,
              w.S, x.K, w.K, cout, w.rows, pair);
    return SCY_ERR_ARG;
  }
  switch (x.S) {
    case 3: return launch_variant<3, T>(x, w, D, ldd, cout, s, status, rps, bit, pair);
    case 4: return launch_variant<4, T>(x, w, D, ldd, cout, s, status, rps, bit, pair);
    case 5: return launch_variant<5, T>(x, w, D, ldd, cout, s, status, rps, bit, pair);
    case 6: return launch_variant<6, T>(x, w, D, ldd, cout, s, status, rps, bit, 0);
    case 7: return launch_variant<7, T>(x, w, D, ldd, cout, s, status, rps, bit, 0);
    default: break;
  }
  set_error("ozk_gemm: %d digit planes (3 to 7 are built)", x.S);
  return SCY_ERR_ARG;
}

}  // namespace

int ozk_cols_per_tile(int S) { return ozk_cn(S); }
int ozk_cols_per_tile_pair(int S) { return S <= 5 ? ozk_cn(S, 1) : 0; }

int ozk_prepare(int S) {
  switch (S) {
    case 3: return prepare_s<3>();
    case 4: return prepare_s<4>();
    case 5: return prepare_s<5>();
    case 6: return prepare_s<6>();
    case 7: return prepare_s<7>();
    default: break;
  }
  set_error("ozk_prepare: %d digit planes (3 to 7 are built)", S);
  return SCY_ERR_ARG;
}

int OzkOperand::alloc_weights(int S_, int rows_, int K_, int esz_) {
  SCY_TRY(alloc(S_, rows_, K_, ozk_cols_per_tile(S_), esz_));
  box_rows_pair = ozk_cols_per_tile_pair(S_);
  if (box_rows_pair > 0 &&
      tma_map_3d_sw64(&map_pair, dig.p, esz == 2 ? CU_TENSOR_MAP_DATA_TYPE_UINT16 : CU_TENSOR_MAP_DATA_TYPE_UINT8,
                      Kp, rows, S, Kp * esz, plane * esz, OZK_BK / esz, box_rows_pair, S) != SCY_OK)
    return SCY_ERR_CUDA;
  return SCY_OK;
}

bool ozk_bf16_exact(int S, int K) {
  const long Kp = (K + 15) / 16 * 16;
  return (long)S * 64 * 64 * Kp < (1L << 24);
}

int OzkOperand::alloc(int S_, int rows_, int K_, int box_rows_, int esz_) {
  if (S_ < 3 || S_ > 7 || rows_ < 1 || K_ < 1 || K_ > 1024 || box_rows_ < 8 || box_rows_ > 256 ||
      (esz_ != 1 && esz_ != 2) || (esz_ == 2 && !ozk_bf16_exact(S_, K_))) {
    set_error("OzkOperand: invalid shape (S %d, rows %d, K %d, box rows %d, digit bytes %d)", S_, rows_, K_,
              box_rows_, esz_);
    return SCY_ERR_ARG;
  }
  S = S_;
  rows = rows_;
  K = K_;
  esz = esz_;
  const int kq = OZK_BK / esz;  // digits per 64-byte stage row (the TMA box; zero-filled past Kp)
  const int ke = 32 / esz;      // digits per MMA K step
  Kp = (K + ke - 1) / ke * ke;
  box_rows = box_rows_;
  plane = (long)rows * Kp;
  SCY_TRY(dig.alloc((size_t)S * plane * esz));
  SCY_TRY(expo.alloc((size_t)rows * sizeof(int)));
  // zero once: the K padding of every row stays zero
  SCY_CUDA_TRY(cudaMemset(dig.p, 0, (size_t)S * plane * esz));
  SCY_CUDA_TRY(cudaMemset(expo.p, 0, (size_t)rows * sizeof(int)));
  if (tma_map_3d_sw64(&map, dig.p, esz == 2 ? CU_TENSOR_MAP_DATA_TYPE_UINT16 : CU_TENSOR_MAP_DATA_TYPE_UINT8, Kp,
                      rows, S, Kp * esz, plane * esz, kq, box_rows, S) != SCY_OK)
    return SCY_ERR_CUDA;
  return SCY_OK;
}

template <typename Tin, int BF>
static void launch_split_reg(OzkOperand& o, const Tin* X, long ldx, cudaStream_t s, int blocks) {
  unsigned char* d = o.dig.as<unsigned char>();
  int* ex = o.expo.as<int>();
  if (o.Kp <= 128)
    ozk_split_reg_kernel<Tin, BF, 1><<<blocks, 256, 0, s>>>(X, ldx, o.rows, o.K, o.Kp, o.S, d, o.plane, ex);
  else if (o.Kp <= 256)
    ozk_split_reg_kernel<Tin, BF, 2><<<blocks, 256, 0, s>>>(X, ldx, o.rows, o.K, o.Kp, o.S, d, o.plane, ex);
  else if (o.Kp <= 512)
    ozk_split_reg_kernel<Tin, BF, 4><<<blocks, 256, 0, s>>>(X, ldx, o.rows, o.K, o.Kp, o.S, d, o.plane, ex);
  else
    ozk_split_reg_kernel<Tin, BF, 8><<<blocks, 256, 0, s>>>(X, ldx, o.rows, o.K, o.Kp, o.S, d, o.plane, ex);
}

template <typename Tin>
static int split_any(OzkOperand& o, const Tin* X, long ldx, cudaStream_t s) {
  const int threads = 256;
  const int blocks = (int)(((long)o.rows * 32 + threads - 1) / threads);
  if (o.Kp <= 1024) {  // the row in registers
    if (o.esz == 2)
      launch_split_reg<Tin, 1>(o, X, ldx, s, blocks);
    else
      launch_split_reg<Tin, 0>(o, X, ldx, s, blocks);
    SCY_LAUNCH_CHECK();
    return SCY_OK;
  }
  if (o.esz == 2)
    ozk_split_kernel<Tin, 1><<<blocks, threads, 0, s>>>(X, ldx, o.rows, o.K, o.Kp, o.S, o.dig.as<unsigned char>(),
                                                        o.plane, o.expo.as<int>());
  else
    ozk_split_kernel<Tin, 0><<<blocks, threads, 0, s>>>(X, ldx, o.rows, o.K, o.Kp, o.S, o.dig.as<unsigned char>(),
                                                        o.plane, o.expo.as<int>());
  SCY_LAUNCH_CHECK();
  return SCY_OK;
}

int ozk_split(OzkOperand& o, const double* X, long ldx, cudaStream_t s) { return split_any(o, X, ldx, s); }
int ozk_split(OzkOperand& o, const float* X, long ldx, cudaStream_t s) { return split_any(o, X, ldx, s); }

int ozk_set_host(OzkOperand& o, const double* W, long ldw, cudaStream_t s) {
  std::vector<int8_t> dig((size_t)o.S * o.plane, 0);
  std::vector<uint16_t> dig2(o.esz == 2 ? (size_t)o.S * o.plane : 0, 0);
  std::vector<int> ex(o.rows, 0);
  for (int r = 0; r < o.rows; ++r) {
    const double* x = W + (long)r * ldw;
    double m = 0.0;
    for (int k = 0; k < o.K; ++k) m = std::fmax(m, std::fabs(x[k]));
    const int e = m > 0.0 ? std::ilogb(m) + 2 : 0;
    ex[r] = e;
    for (int k = 0; k < o.K; ++k) {
      double t = std::ldexp(x[k], 7 - e);
      for (int i = 0; i < o.S; ++i) {
        const double d = std::nearbyint(t);
        t = (t - d) * 128.0;
        const size_t at = (size_t)i * o.plane + (size_t)r * o.Kp + k;
        if (o.esz == 2) {
          // bf16 pattern of the integer digit: the upper half of its FP32 pattern
          const float f = (float)d;
          uint32_t u;
          std::memcpy(&u, &f, 4);
          dig2[at] = (uint16_t)(u >> 16);
        } else {
          dig[at] = (int8_t)(int)d;
        }
      }
    }
  }
  if (o.esz == 2)
    SCY_CUDA_TRY(cudaMemcpyAsync(o.dig.p, dig2.data(), dig2.size() * 2, cudaMemcpyHostToDevice, s));
  else
    SCY_CUDA_TRY(cudaMemcpyAsync(o.dig.p, dig.data(), dig.size(), cudaMemcpyHostToDevice, s));
  SCY_CUDA_TRY(cudaMemcpyAsync(o.expo.p, ex.data(), ex.size() * sizeof(int), cudaMemcpyHostToDevice, s));
  SCY_CUDA_TRY(cudaStreamSynchronize(s));
  return SCY_OK;
}

int ozk_gemm(const OzkOperand& x, const OzkOperand& w, double* D, long ldd, int cout, cudaStream_t s,
             unsigned* status, int rows_per_status, unsigned bit, int pair) {
  return gemm_any<double>(x, w, D, ldd, cout, s, status, rows_per_status, bit, pair);
}

int ozk_gemm(const OzkOperand& x, const OzkOperand& w, float* D, long ldd, int cout, cudaStream_t s,
             unsigned* status, int rows_per_status, unsigned bit, int pair) {
  return gemm_any<float>(x, w, D, ldd, cout, s, status, rows_per_status, bit, pair);
}

}  // namespace scy

// ---------------------------------------------------------------------------
// C ABI: the product on its own (set-up and digit planes allocated per call)
extern "C" scy_status scy_ozaki_matmul(const double* X, long ldx, int rows, int K, const double* W, long ldw,
                                       int cols, int S, double* D, long ldd, int ctas_per_sm, int bf16_digits) {
  using namespace scy;
  if (!X || !W || !D || rows < 1 || cols < 1 || K < 1 || ldx < K || ldw < K || ldd < cols ||
      (ctas_per_sm < 0 || ctas_per_sm > 2) || (ctas_per_sm != 1 && S > 5) ||
      (bf16_digits && !ozk_bf16_exact(S, K))) {
    set_error("scy_ozaki_matmul: invalid arguments");
    return SCY_ERR_ARG;
  }
  const int esz = bf16_digits ? 2 : 1;
  OzkOperand x, w;
  SCY_TRY(x.alloc(S, rows, K, 128, esz));
  SCY_TRY(w.alloc_weights(S, cols, K, esz));
  cudaStream_t s = 0;
  SCY_TRY(ozk_set_host(w, W, ldw, s));
  SCY_TRY(ozk_split(x, X, ldx, s));
  DevBuf status;
  SCY_TRY(status.alloc(sizeof(unsigned)));
  SCY_CUDA_TRY(cudaMemsetAsync(status.p, 0, sizeof(unsigned), s));
  SCY_TRY(ozk_gemm(x, w, D, ldd, cols, s, status.as<unsigned>(), 1 << 30, 1u,
                   ctas_per_sm == 2 ? 1 : ctas_per_sm == 0 ? 2 : 0));
  unsigned st = 0;
  SCY_CUDA_TRY(cudaMemcpyAsync(&st, status.p, sizeof(unsigned), cudaMemcpyDeviceToHost, s));
  SCY_CUDA_TRY(cudaStreamSynchronize(s));
  if (st) {
    set_error("scy_ozaki_matmul: a pipeline wait in the product kernel ran out");
    return SCY_ERR_CUDA;
  }
  return SCY_OK;
}
