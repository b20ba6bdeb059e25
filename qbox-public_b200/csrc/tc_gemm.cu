// tcgen05 split-precision GEMM for sm_100a.
//
//   D(m, n) = sum_k A(k, m) B(k, n)   over the three split terms
//             A_hi B_hi + A_hi B_lo + A_lo B_hi   (FP32 accumulate)
//
// in two operand kinds: BF16 splits (kind::f16, 16 significant bits) for
// the inner products over the plane-wave rows, and TF32 splits
// (kind::tf32, 22 bits) for the tall updates.
//
// A and B are K-major (column-major with the contraction index contiguous),
// as the wavefunction and projector matrices of a SlaterDet are.  The inner
// products of the electronic step (projections F = A_nl^T C, the residual
// C^T (H C), the overlaps C^T C and C^T C_last) use the BF16 kind with split
// K and an FP64 sum of the partials.  The tall updates H C += A_nl F,
// H C -= C A and C -= C (I - X) contract over bands or projectors: their A
// operand is the transposed split of A_nl or C (bands contiguous), and the
// epilogue adds alpha * D into the FP64 output directly.
//
// One CTA computes a 128 x 128 FP32 tile of one split-K slice:
//   warp 0  - TMA producer: per 64-wide K block one pipeline stage receives
//             the four 128x64 BF16 tiles A_hi, A_lo, B_hi, B_lo
//             (128-byte swizzle); mbarrier expect_tx per stage;
//   warp 1  - allocates 128 TMEM columns; one elected thread issues the
//             12 tcgen05.mma (3 terms x 4 K-steps of 16) per stage and
//             commits the stage back to the producer;
//   warps 4-7 - epilogue: tcgen05.ld of the accumulator (each warp its 32
//             TMEM lanes) and coalesced FP32 stores of the partial tile.
// Split-K partials are summed in FP64 by k_reduce_splits2d.  Every
// mbarrier wait is bounded; a wait that runs out sets an error flag that
// the host turns into an error, and the CTA still releases its TMEM.
#include <cuda.h>
#include <cuda_bf16.h>

#include <algorithm>
#include <cstdint>

#include "qbx_internal.h"

namespace qbx {

namespace tc {

constexpr int BM = 128, BN = 128;
constexpr int KIND_BF16 = 0, KIND_TF32 = 1;
// K elements per 128-byte tile row: 64 BF16 or 32 TF32
__host__ __device__ constexpr int bk_of(int kind) { return kind == KIND_BF16 ? 64 : 32; }
constexpr int BK = 64;                            // BF16 (kept for callers' checks)
constexpr int STAGES = 3;
constexpr int TILE_BYTES = BM * 128;              // 16 KB per operand tile
constexpr int STAGE_BYTES = 4 * TILE_BYTES;       // A_hi, A_lo, B_hi, B_lo
constexpr int SMEM_BYTES = STAGES * STAGE_BYTES + 1024 /* align */ + 256 /* barriers */;
// warps 0-3: TMA producer, MMA issuer, two idle; then EPW epilogue warps,
// EPW/4 per TMEM lane quarter (warp w reads lanes 32*(w%4) .. 32*(w%4)+31),
// each holding BN*4/EPW columns of the tile
__host__ __device__ constexpr int threads_of(int epw) { return 128 + 32 * epw; }
// TMEM: two hi*hi accumulators used in turn (256 columns); with the
// correction terms kept apart (sep), two more for hi*lo + lo*hi (512 columns)
__host__ __device__ constexpr uint32_t tmem_cols_of(int sep) { return sep ? 4 * BN : 2 * BN; }
constexpr long long WAIT_LIMIT = 1ll << 24;       // bounded spins per wait

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
}

// bounded wait for the phase with the given parity to complete
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
  const uint32_t a = smem_u32(bar);
  for (long long it = 0; it < WAIT_LIMIT; ++it) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, uint64_t* bar,
                                            int x, int y) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes "
      "[%0], [%1, {%3, %4}], [%2];" ::"r"(smem_u32(dst)),
      "l"((uint64_t)map), "r"(smem_u32(bar)), "r"(x), "r"(y)
      : "memory");
}

// K-major operand tile in shared memory, 128-byte swizzle, rows of 128 bytes,
// 8-row groups 1024 bytes apart (the canonical UMMA K-major SW128 layout).
__device__ __forceinline__ uint64_t smem_desc(const void* tile) {
  const uint64_t addr = smem_u32(tile);
  return ((addr & 0x3FFFF) >> 4) | (1ull << 16) | (64ull << 32) | (1ull << 46) | (2ull << 61);
}

// MN-major operand tile (M contiguous): boxes of 128 bytes of M by the K
// block, each K row one 128-byte swizzled row; BF16 tiles in 8-row groups
// 1024 bytes apart (stride byte offset), the boxes (128 bytes of M each)
// `box_bytes` apart (leading byte offset).
// TF32 tiles use the 128-byte swizzle with 32-byte atoms (layout type 1):
// groups of 4 K rows, 512 bytes apart.
template <int KIND>
__device__ __forceinline__ uint64_t smem_desc_mn(const void* tile, uint32_t box_bytes) {
  const uint64_t addr = smem_u32(tile);
  constexpr uint64_t sbo = KIND == KIND_BF16 ? 1024 : 512;
  constexpr uint64_t layout = KIND == KIND_BF16 ? 2 : 1;
  return ((addr & 0x3FFFF) >> 4) | ((uint64_t)(box_bytes >> 4) << 16) | ((sbo >> 4) << 32) |
         (1ull << 46) | (layout << 61);
}

// Instruction descriptor: F32 accumulate (bits 4-5 = 1), A and B formats
// (bits 7-9, 10-12: BF16 = 1 for kind::f16, TF32 = 2 for kind::tf32), both
// K-major, N >> 3 at bit 17, M >> 4 at bit 24.
__host__ __device__ constexpr uint32_t idesc_of(int kind) {
  const uint32_t fmt = kind == KIND_BF16 ? 1u : 2u;
  return (1u << 4) | (fmt << 7) | (fmt << 10) | ((uint32_t)(BN >> 3) << 17) |
         ((uint32_t)(BM >> 4) << 24);
}

template <int KIND>
__device__ __forceinline__ void umma(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t acc) {
  if constexpr (KIND == KIND_BF16) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
        "l"(da), "l"(db), "r"(idesc_of(KIND_BF16)), "r"(acc)
        : "memory");
  } else {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
        "l"(da), "l"(db), "r"(idesc_of(KIND_TF32)), "r"(acc)
        : "memory");
  }
}

// 16 consecutive TMEM columns of this warp's 32 lanes (one per thread);
// the caller waits with tcgen05.wait::ld before reading r
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t* r) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
      "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
        "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ void umma_commit(uint64_t* bar) {
  asm volatile(
      "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
          smem_u32(bar))
      : "memory");
}

// Accumulation: the MMA warp fills one of two 128-column TMEM accumulators
// with `chunk` K blocks (64 * chunk products of each split term per
// element) and commits it; the epilogue warps add that accumulator into FP32
// registers (round to nearest) and hand it back, while the MMA warp fills
// the other one.  The tensor core's own FP32 additions into TMEM do not
// round to nearest: each one can shift the running sum toward zero by up to
// an ulp, so a long chain biases a coherent inner product low (at 145 838
// rows and 96 additions per chain that bias reached 1.7e-6 of F = A^T C,
// 3e-6 of E_nl).  Short chains keep that bias down.  With corr_mul > 0 the
// small terms hi*lo + lo*hi (2^-8 of the sum) go to a second pair of
// accumulators whose chains are corr_mul times longer, so that the large
// hi*hi chain carries one MMA per K step of 16 and the epilogue drains the
// small terms only every corr_mul chunks.
// Output: with ws != nullptr the FP32 tile of split-K slice z goes to
// ws[z][col * M + row]; otherwise (no K split) C[col * ldc + row] =
// alpha * D + beta * C in FP64.  Rows >= M and columns >= N are not stored.
template <int KIND, int EPW>
__global__ void __launch_bounds__(threads_of(EPW), 1)
k_tc_split_gemm(const __grid_constant__ CUtensorMap ma_hi, const __grid_constant__ CUtensorMap ma_lo,
                const __grid_constant__ CUtensorMap mb_hi, const __grid_constant__ CUtensorMap mb_lo,
                int M, int N, int nkb, int kb_per_split, float* __restrict__ ws,
                double* __restrict__ C, int ldc, double alpha, double beta,
                int* __restrict__ err, int lower, int chunk, int corr_mul) {
  // lower: a tile whose every column is right of its every row holds only
  // the strict upper triangle and is not formed (the whole CTA leaves before
  // it allocates anything)
  {
    const int tm0 = (ws ? blockIdx.x : blockIdx.y) * BM, tn0 = (ws ? blockIdx.y : blockIdx.x) * BN;
    if (lower && tn0 >= tm0 + BM) return;
  }
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  unsigned char* base = (unsigned char*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  uint64_t* full = (uint64_t*)(base + STAGES * STAGE_BYTES);
  uint64_t* empty = full + STAGES;
  uint64_t* tfull = empty + STAGES;      // accumulator b filled
  uint64_t* tfree = tfull + 2;           // accumulator b drained by the epilogue
  uint64_t* cfull = tfree + 2;           // correction accumulator b filled
  uint64_t* cfree = cfull + 2;           // correction accumulator b drained
  uint32_t* tmem_slot = (uint32_t*)(cfree + 2);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  // without a K split the N tiles of one M tile are adjacent in the grid, so
  // the CTAs that share an A tile run together and A streams from HBM once
  const int m0 = (ws ? blockIdx.x : blockIdx.y) * BM, n0 = (ws ? blockIdx.y : blockIdx.x) * BN;
  const int kb0 = blockIdx.z * kb_per_split;
  const int kb1 = min(nkb, kb0 + kb_per_split);
  const int niter = max(0, kb1 - kb0);
  const int nchunk = (niter + chunk - 1) / chunk;
  const int sep = corr_mul > 0 ? 1 : 0;
  const int cchunk = chunk * (sep ? corr_mul : 1);   // K blocks per correction chain
  const uint32_t tmem_cols = tmem_cols_of(sep);

  if (threadIdx.x == 0) {
    for (int s = 0; s < STAGES; s++) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    for (int b = 0; b < 2; b++) {
      mbar_init(&tfull[b], 1);
      mbar_init(&tfree[b], EPW);         // one arrival per epilogue warp
      mbar_init(&cfull[b], 1);
      mbar_init(&cfree[b], EPW);
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(tmem_slot)),
                 "r"(tmem_cols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tmem_slot;

  if (warp == 0 && lane == 0) {
    // ---------------- TMA producer
    for (int it = 0; it < niter; ++it) {
      const int s = it % STAGES;
      const uint32_t ph = (uint32_t)((it / STAGES) & 1);
      if (!mbar_wait(&empty[s], ph ^ 1u)) { atomicExch(err, 1); break; }
      unsigned char* st = base + s * STAGE_BYTES;
      mbar_expect_tx(&full[s], STAGE_BYTES);
      const int kx = (kb0 + it) * bk_of(KIND);
      tma_load_2d(st + 0 * TILE_BYTES, &ma_hi, &full[s], kx, m0);
      tma_load_2d(st + 1 * TILE_BYTES, &ma_lo, &full[s], kx, m0);
      tma_load_2d(st + 2 * TILE_BYTES, &mb_hi, &full[s], kx, n0);
      tma_load_2d(st + 3 * TILE_BYTES, &mb_lo, &full[s], kx, n0);
    }
  } else if (warp == 1 && lane == 0) {
    // ---------------- MMA issuer
    for (int it = 0; it < niter; ++it) {
      const int c = it / chunk, b = c & 1;
      const int cc = it / cchunk, cb = cc & 1;
      const bool chunk_start = (it % chunk) == 0;
      const bool corr_start = (it % cchunk) == 0;
      if (chunk_start && c >= 2 && !mbar_wait(&tfree[b], (uint32_t)(((c >> 1) - 1) & 1))) {
        atomicExch(err, 4);
        break;
      }
      if (sep && corr_start && cc >= 2 &&
          !mbar_wait(&cfree[cb], (uint32_t)(((cc >> 1) - 1) & 1))) {
        atomicExch(err, 5);
        break;
      }
      const int s = it % STAGES;
      const uint32_t ph = (uint32_t)((it / STAGES) & 1);
      if (!mbar_wait(&full[s], ph)) { atomicExch(err, 2); break; }
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      unsigned char* st = base + s * STAGE_BYTES;
      const uint64_t dah = smem_desc(st + 0 * TILE_BYTES);
      const uint64_t dal = smem_desc(st + 1 * TILE_BYTES);
      const uint64_t dbh = smem_desc(st + 2 * TILE_BYTES);
      const uint64_t dbl = smem_desc(st + 3 * TILE_BYTES);
      const uint32_t tacc = tmem + (uint32_t)(b * BN);
      const uint32_t tcor = sep ? tmem + (uint32_t)((2 + cb) * BN) : tacc;
      // 4 MMAs of 32 bytes of K each (16 BF16 or 8 TF32)
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        const uint64_t off = (uint64_t)(k * 32) >> 4;
        const uint32_t accumulate = (chunk_start && k == 0) ? 0u : 1u;
        const uint32_t cacc = sep ? ((corr_start && k == 0) ? 0u : 1u) : 1u;
        umma<KIND>(tacc, dah + off, dbh + off, accumulate);
        umma<KIND>(tcor, dah + off, dbl + off, cacc);
        umma<KIND>(tcor, dal + off, dbh + off, 1u);
      }
      umma_commit(&empty[s]);
      if ((it % chunk) == chunk - 1 || it == niter - 1) umma_commit(&tfull[b]);
      if (sep && ((it % cchunk) == cchunk - 1 || it == niter - 1)) umma_commit(&cfull[cb]);
    }
  } else if (warp >= 4) {
    // ---------------- epilogue: drain each chunk into FP32 registers
    constexpr int COLS = BN * 4 / EPW;             // columns of this warp
    const int wq = warp & 3;                       // TMEM lanes 32*wq .. 32*wq+31
    const int cbase = ((warp - 4) >> 2) * COLS;    // first column of this warp
    const int row = m0 + wq * 32 + lane;
    const uint32_t tlane = tmem + ((uint32_t)(wq * 32) << 16) + (uint32_t)cbase;
    float acc[COLS];
#pragma unroll
    for (int j = 0; j < COLS; ++j) acc[j] = 0.0f;
    // acc += this warp's columns of one accumulator, 64 columns (four loads
    // in flight) per wait
    auto drain = [&](uint32_t col0) {
#pragma unroll
      for (int c0 = 0; c0 < COLS; c0 += 64) {
        uint32_t r[64];
#pragma unroll
        for (int q = 0; q < 4; ++q) tmem_ld16(tlane + col0 + (uint32_t)(c0 + 16 * q), r + 16 * q);
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
        for (int j = 0; j < 64; ++j) acc[c0 + j] += __uint_as_float(r[j]);
      }
    };
    bool ok = true;
    for (int c = 0; c < nchunk && ok; ++c) {
      const int b = c & 1;
      if (!mbar_wait(&tfull[b], (uint32_t)((c >> 1) & 1))) {
        atomicExch(err, 3);
        ok = false;
        break;
      }
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      drain((uint32_t)(b * BN));
      asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
      __syncwarp();
      if (lane == 0) mbar_arrive(&tfree[b]);
      if (sep && ((c + 1) % corr_mul == 0 || c == nchunk - 1)) {
        const int cc = c / corr_mul, cb = cc & 1;
        if (!mbar_wait(&cfull[cb], (uint32_t)((cc >> 1) & 1))) {
          atomicExch(err, 6);
          ok = false;
          break;
        }
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        drain((uint32_t)((2 + cb) * BN));
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        __syncwarp();
        if (lane == 0) mbar_arrive(&cfree[cb]);
      }
    }
    if (ws) {
      float* out = ws + (size_t)blockIdx.z * M * N;
      if (row < M) {
#pragma unroll
        for (int j = 0; j < COLS; ++j) {
          const int col = n0 + cbase + j;
          if (col < N) out[(size_t)col * M + row] = ok ? acc[j] : 0.0f;
        }
      }
    } else if (row < M && ok) {
      double* crow = C + row;
      if (beta == 1.0) {
        // C += alpha D: fire-and-forget FP64 adds (each element has one
        // writer, so the result does not depend on their order); no load
        // round trips in the epilogue
#pragma unroll
        for (int j = 0; j < COLS; ++j) {
          const int col = n0 + cbase + j;
          if (col < N) atomicAdd(crow + (size_t)col * ldc, alpha * (double)acc[j]);
        }
      } else {
      // FP64 read-modify-write of the tile, 16 columns per group: the
      // group's loads are issued together so their latencies overlap (one
      // load at a time would leave the epilogue waiting 128 round trips)
      constexpr int G = 16;
#pragma unroll
      for (int j0 = 0; j0 < COLS; j0 += G) {
        double old[G];
        if (beta != 0.0) {
#pragma unroll
          for (int j = 0; j < G; ++j) {
            const int col = n0 + cbase + j0 + j;
            old[j] = col < N ? crow[(size_t)col * ldc] : 0.0;
          }
        }
#pragma unroll
        for (int j = 0; j < G; ++j) {
          const int col = n0 + cbase + j0 + j;
          if (col < N)
            crow[(size_t)col * ldc] = alpha * (double)acc[j0 + j] + (beta != 0.0 ? beta * old[j] : 0.0);
        }
      }
      }
    }
  }
  __syncthreads();
  if (warp == 1) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                 "r"(tmem_cols)
                 : "memory");
  }
}

// ------------------------------------------------------------ CTA pairs
// The same product on 256 x 128 tiles, computed by a cluster of two CTAs on
// two SMs with tcgen05.mma.cta_group::2.  CTA r of the pair loads its own 128
// rows of A and half of B's 128 columns (columns 64 r .. 64 r + 63) into its
// shared memory; the pair's first CTA issues the MMAs, which read A and B
// from both CTAs' shared memory and accumulate rows 128 r .. 128 r + 127 of
// the tile in CTA r's TMEM.  Per SM a K block moves 48 KB of operands
// instead of 64 KB, the MMAs read a quarter less from each SM's shared
// memory, and four pipeline stages fit.
//   - both CTAs' TMA loads complete on the first CTA's stage barrier, whose
//     expected bytes the first CTA sets for the pair;
//   - the first CTA's MMA commits arrive on the same barrier of both CTAs
//     (stage free, accumulator filled);
//   - the epilogue warps of both CTAs drain their own TMEM and hand the
//     accumulator back on the first CTA's barrier.
// The accumulation chains, the epilogue and the outputs are those of
// k_tc_split_gemm.  Every mbarrier wait is bounded; both CTAs meet at a
// cluster barrier after the barriers are set up and again before TMEM is
// freed, and every path (a timed-out wait included) reaches both.
// The pair's tile is 256 rows by BNT = 128 or 256 columns; each CTA holds
// BNT / 2 rows of B per stage.  With BNT = 256 two accumulators fill the 512
// TMEM columns, so the correction terms share the hi*hi chain (corr_mul 0).
template <int BNT> struct PairCfg {
  static constexpr int HALF_BYTES = (BNT / 2) * 128;                     // 8 or 16 KB
  static constexpr int STAGE_BYTES = 2 * TILE_BYTES + 2 * HALF_BYTES;   // 48 or 64 KB
  static constexpr int STAGES = BNT == 128 ? 4 : 3;
  static constexpr int SMEM_BYTES = STAGES * STAGE_BYTES + 1024 + 256;
};

// instruction descriptor of the pair's 256 x BNT MMA; amn: A is MN-major
// (bit 15)
__host__ __device__ constexpr uint32_t idesc_pair_of(int kind, int bnt, bool amn = false) {
  const uint32_t fmt = kind == KIND_BF16 ? 1u : 2u;
  return (1u << 4) | (fmt << 7) | (fmt << 10) | ((amn ? 1u : 0u) << 15) |
         ((uint32_t)(bnt >> 3) << 17) | ((uint32_t)((2 * BM) >> 4) << 24);
}

__device__ __forceinline__ uint32_t cluster_rank() {
  uint32_t r;
  asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
  return r;
}

// shared::cluster address of this shared variable in CTA `rank` of the cluster
__device__ __forceinline__ uint32_t cluster_addr(const void* p, uint32_t rank) {
  uint32_t r;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(smem_u32(p)), "r"(rank));
  return r;
}

__device__ __forceinline__ void cluster_sync_all() {
  asm volatile(
      "barrier.cluster.arrive.release.aligned;\n\t"
      "barrier.cluster.wait.acquire.aligned;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_remote(uint32_t addr) {
  asm volatile("mbarrier.arrive.release.cluster.shared::cluster.b64 _, [%0];" ::"r"(addr)
               : "memory");
}

// bounded wait, acquiring at cluster scope (the barrier's arrivals come from
// the other CTA of the pair or from the pair's MMAs)
__device__ __forceinline__ bool mbar_wait_cluster(uint64_t* bar, uint32_t parity) {
  const uint32_t a = smem_u32(bar);
  for (long long it = 0; it < WAIT_LIMIT; ++it) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.acquire.cluster.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

// TMA load into this CTA's shared memory, its bytes counted on the pair's
// barrier at cluster address bar (each CTA loads only its own tiles from this
// GPU's memory)
__device__ __forceinline__ void tma_load_2d_pair(void* dst, const CUtensorMap* map, uint32_t bar,
                                                 int x, int y) {
  asm volatile(
      "cp.async.bulk.tensor.2d.cta_group::2.shared::cluster.global.mbarrier::complete_tx::bytes "
      "[%0], [%1, {%3, %4}], [%2];" ::"r"(smem_u32(dst)),
      "l"((uint64_t)map), "r"(bar), "r"(x), "r"(y)
      : "memory");
}

template <int KIND, int BNT, bool AMN = false>
__device__ __forceinline__ void umma_pair(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t acc) {
  if constexpr (KIND == KIND_BF16) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::2.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
        "l"(da), "l"(db), "r"(idesc_pair_of(KIND_BF16, BNT, AMN)), "r"(acc)
        : "memory");
  } else {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::2.kind::tf32 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
        "l"(da), "l"(db), "r"(idesc_pair_of(KIND_TF32, BNT, AMN)), "r"(acc)
        : "memory");
  }
}

// one arrival on the barrier at this offset in both CTAs of the pair when
// the MMAs issued so far have completed
__device__ __forceinline__ void umma_commit_pair(uint64_t* bar) {
  asm volatile(
      "{\n\t.reg .b16 m;\n\t"
      "mov.b16 m, 3;\n\t"
      "tcgen05.commit.cta_group::2.mbarrier::arrive::one.shared::cluster.multicast::cluster.b64 "
      "[%0], m;\n\t}" ::"r"(smem_u32(bar))
      : "memory");
}

// AMN: A is MN-major in global memory (its M rows contiguous, as the
// columns of a SlaterDet are): the tall updates then read the plain split of
// the wavefunction block instead of a transposed copy.  Its 128 rows per K
// block arrive as boxes of 128 bytes of M.
template <int KIND, int EPW, int BNT, bool AMN>
__global__ void __launch_bounds__(threads_of(EPW), 1)
k_tc_pair_gemm(const __grid_constant__ CUtensorMap ma_hi, const __grid_constant__ CUtensorMap ma_lo,
               const __grid_constant__ CUtensorMap mb_hi, const __grid_constant__ CUtensorMap mb_lo,
               int M, int N, int nkb, int kb_per_split, float* __restrict__ ws,
               double* __restrict__ C, int ldc, double alpha, double beta,
               int* __restrict__ err, int lower, int chunk, int corr_mul) {
  // the pair is M tiles 2p and 2p + 1, CTA ranks 0 and 1 of a cluster along
  // x.  Without a K split, x runs over (N tile, rank) and y over the pairs,
  // so the N tiles that share a pair's A tiles run together and A streams
  // from HBM once.
  const int mt = ws ? (int)blockIdx.x : 2 * (int)blockIdx.y + (int)(blockIdx.x & 1);
  const int nt = ws ? (int)blockIdx.y : (int)(blockIdx.x >> 1);
  using P = PairCfg<BNT>;
  // A descriptors and the step of one MMA's K slice (32 bytes of K within a
  // K-major row; 16 or 8 rows of 128 bytes down an MN-major tile), in the
  // descriptor's 16-byte address units
  constexpr uint32_t A_BOX = AMN ? TILE_BYTES / (BM / (128 / (KIND == KIND_BF16 ? 2 : 4))) : 0;
  auto a_desc = [](const void* t) { return AMN ? smem_desc_mn<KIND>(t, A_BOX) : smem_desc(t); };
  constexpr uint64_t AK = AMN ? (uint64_t)(KIND == KIND_BF16 ? 16 : 8) * 128 / 16 : 32 / 16;
  const int m0 = mt * BM, n0 = nt * BNT;
  // lower: a pair whose every row lies above the tile's first column holds
  // only the strict upper triangle; both CTAs leave before anything is set up
  if (lower && n0 >= (mt & ~1) * BM + 2 * BM) return;
  const uint32_t rank = cluster_rank();
  const bool lead = rank == 0;
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  unsigned char* base = (unsigned char*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  uint64_t* full = (uint64_t*)(base + P::STAGES * P::STAGE_BYTES);
  uint64_t* empty = full + P::STAGES;
  uint64_t* tfull = empty + P::STAGES;
  uint64_t* tfree = tfull + 2;
  uint64_t* cfull = tfree + 2;
  uint64_t* cfree = cfull + 2;
  uint32_t* tmem_slot = (uint32_t*)(cfree + 2);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int kb0 = blockIdx.z * kb_per_split;
  const int kb1 = min(nkb, kb0 + kb_per_split);
  const int niter = max(0, kb1 - kb0);
  const int sep = corr_mul > 0 ? 1 : 0;
  const int nchunk = (niter + chunk - 1) / chunk;
  const int cchunk = chunk * (sep ? corr_mul : 1);
  const uint32_t tmem_cols = (uint32_t)(sep ? 4 * BNT : 2 * BNT);

  if (threadIdx.x == 0) {
    for (int s = 0; s < P::STAGES; s++) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    for (int b = 0; b < 2; b++) {
      mbar_init(&tfull[b], 1);
      mbar_init(&tfree[b], 2 * EPW);    // the epilogue warps of both CTAs
      mbar_init(&cfull[b], 1);
      mbar_init(&cfree[b], 2 * EPW);
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::2.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(tmem_slot)),
                 "r"(tmem_cols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::2.sync.aligned;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  }
  __syncthreads();
  cluster_sync_all();   // both CTAs' barriers exist before any arrival crosses the pair
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tmem_slot;

  if (warp == 0 && lane == 0) {
    // ---------------- TMA producer (both CTAs)
    bool ok = true;
    for (int it = 0; it < niter; ++it) {
      const int s = it % P::STAGES;
      const uint32_t ph = (uint32_t)((it / P::STAGES) & 1);
      if (!mbar_wait_cluster(&empty[s], ph ^ 1u)) {
        atomicExch(err, 1);
        ok = false;
        break;
      }
      unsigned char* st = base + s * P::STAGE_BYTES;
      const uint32_t fb = cluster_addr(&full[s], 0);
      if (lead) mbar_expect_tx(&full[s], 2 * P::STAGE_BYTES);
      const int kx = (kb0 + it) * bk_of(KIND);
      const int nb = n0 + (int)rank * (BNT / 2);
      if constexpr (AMN) {
        // M boxes of 128 bytes: 64 BF16 or 32 TF32 rows, K block deep
        constexpr int MW = 128 / (KIND == KIND_BF16 ? 2 : 4);
        constexpr int BOX = TILE_BYTES / (BM / MW);
#pragma unroll
        for (int q = 0; q < BM / MW; ++q) {
          tma_load_2d_pair(st + q * BOX, &ma_hi, fb, m0 + q * MW, kx);
          tma_load_2d_pair(st + TILE_BYTES + q * BOX, &ma_lo, fb, m0 + q * MW, kx);
        }
      } else {
        tma_load_2d_pair(st, &ma_hi, fb, kx, m0);
        tma_load_2d_pair(st + TILE_BYTES, &ma_lo, fb, kx, m0);
      }
      tma_load_2d_pair(st + 2 * TILE_BYTES, &mb_hi, fb, kx, nb);
      tma_load_2d_pair(st + 2 * TILE_BYTES + P::HALF_BYTES, &mb_lo, fb, kx, nb);
    }
    // every stage's last release (a commit of the first CTA's MMAs) has
    // arrived here before this CTA can leave
    for (int it = niter; it < niter + P::STAGES && ok; ++it) {
      const int s = it % P::STAGES;
      if (!mbar_wait_cluster(&empty[s], (uint32_t)(((it / P::STAGES) & 1) ^ 1))) {
        atomicExch(err, 7);
        ok = false;
      }
    }
  } else if (warp == 1 && lane == 0 && lead) {
    // ---------------- MMA issuer (first CTA)
    if (!sep) {
      // One accumulator chain per `chunk` K blocks holding all three terms.
      // Each K block issues its small hi*lo and lo*hi products before its
      // hi*hi products, so the chain's first block adds its small terms to a
      // sum 2^8 times smaller than the whole (the TMEM additions truncate,
      // and their error scales with the running sum).
      for (int c = 0; c < nchunk; ++c) {
        const int b = c & 1;
        const int it0 = c * chunk, it1 = min(niter, it0 + chunk);
        if (c >= 2 && !mbar_wait_cluster(&tfree[b], (uint32_t)(((c >> 1) - 1) & 1))) {
          atomicExch(err, 4);
          break;
        }
        const uint32_t tacc = tmem + (uint32_t)(b * BNT);
        uint32_t accumulate = 0u;
        bool ok = true;
        for (int it = it0; it < it1; ++it) {
          const int s = it % P::STAGES;
          if (!mbar_wait_cluster(&full[s], (uint32_t)((it / P::STAGES) & 1))) {
            ok = false;
            break;
          }
          asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
          unsigned char* st = base + s * P::STAGE_BYTES;
          const uint64_t dah = a_desc(st);
          const uint64_t dal = a_desc(st + TILE_BYTES);
          const uint64_t dbh = smem_desc(st + 2 * TILE_BYTES);
          const uint64_t dbl = smem_desc(st + 2 * TILE_BYTES + P::HALF_BYTES);
#pragma unroll
          for (int k = 0; k < 4; ++k) {
            const uint64_t off = (uint64_t)(k * 32) >> 4;
            umma_pair<KIND, BNT, AMN>(tacc, dah + k * AK, dbl + off, accumulate);
            accumulate = 1u;
            umma_pair<KIND, BNT, AMN>(tacc, dal + k * AK, dbh + off, 1u);
          }
#pragma unroll
          for (int k = 0; k < 4; ++k) {
            const uint64_t off = (uint64_t)(k * 32) >> 4;
            umma_pair<KIND, BNT, AMN>(tacc, dah + k * AK, dbh + off, 1u);
          }
          umma_commit_pair(&empty[s]);
        }
        if (!ok) { atomicExch(err, 2); break; }
        umma_commit_pair(&tfull[b]);
      }
    } else
    for (int it = 0; it < niter; ++it) {
      const int c = it / chunk, b = c & 1;
      const int cc = it / cchunk, cb = cc & 1;
      const bool chunk_start = (it % chunk) == 0;
      const bool corr_start = (it % cchunk) == 0;
      if (chunk_start && c >= 2 &&
          !mbar_wait_cluster(&tfree[b], (uint32_t)(((c >> 1) - 1) & 1))) {
        atomicExch(err, 4);
        break;
      }
      if (sep && corr_start && cc >= 2 &&
          !mbar_wait_cluster(&cfree[cb], (uint32_t)(((cc >> 1) - 1) & 1))) {
        atomicExch(err, 5);
        break;
      }
      const int s = it % P::STAGES;
      const uint32_t ph = (uint32_t)((it / P::STAGES) & 1);
      if (!mbar_wait_cluster(&full[s], ph)) { atomicExch(err, 2); break; }
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      unsigned char* st = base + s * P::STAGE_BYTES;
      const uint64_t dah = a_desc(st);
      const uint64_t dal = a_desc(st + TILE_BYTES);
      const uint64_t dbh = smem_desc(st + 2 * TILE_BYTES);
      const uint64_t dbl = smem_desc(st + 2 * TILE_BYTES + P::HALF_BYTES);
      const uint32_t tacc = tmem + (uint32_t)(b * BNT);
      const uint32_t tcor = sep ? tmem + (uint32_t)((2 + cb) * BNT) : tacc;
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        const uint64_t off = (uint64_t)(k * 32) >> 4;
        const uint32_t accumulate = (chunk_start && k == 0) ? 0u : 1u;
        const uint32_t cacc = sep ? ((corr_start && k == 0) ? 0u : 1u) : 1u;
        umma_pair<KIND, BNT, AMN>(tacc, dah + k * AK, dbh + off, accumulate);
        umma_pair<KIND, BNT, AMN>(tcor, dah + k * AK, dbl + off, cacc);
        umma_pair<KIND, BNT, AMN>(tcor, dal + k * AK, dbh + off, 1u);
      }
      umma_commit_pair(&empty[s]);
      if ((it % chunk) == chunk - 1 || it == niter - 1) umma_commit_pair(&tfull[b]);
      if (sep && ((it % cchunk) == cchunk - 1 || it == niter - 1)) umma_commit_pair(&cfull[cb]);
    }
  } else if (warp >= 4) {
    // ---------------- epilogue (both CTAs): drain this CTA's TMEM rows
    constexpr int COLS = BNT * 4 / EPW;
    // TMEM columns per wait: four loads in flight, or one where the tile's
    // register copy leaves no room for more
    constexpr int LDW = (COLS > 64 || EPW > 8) ? 16 : 64;
    const int wq = warp & 3;
    const int cbase = ((warp - 4) >> 2) * COLS;
    const int row = m0 + wq * 32 + lane;
    const uint32_t tlane = tmem + ((uint32_t)(wq * 32) << 16) + (uint32_t)cbase;
    float acc[COLS];
#pragma unroll
    for (int j = 0; j < COLS; ++j) acc[j] = 0.0f;
    auto drain = [&](uint32_t col0) {
#pragma unroll
      for (int c0 = 0; c0 < COLS; c0 += LDW) {
        uint32_t r[LDW];
#pragma unroll
        for (int q = 0; q < LDW / 16; ++q)
          tmem_ld16(tlane + col0 + (uint32_t)(c0 + 16 * q), r + 16 * q);
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
        for (int j = 0; j < LDW; ++j) acc[c0 + j] += __uint_as_float(r[j]);
      }
    };
    bool ok = true;
    for (int c = 0; c < nchunk && ok; ++c) {
      const int b = c & 1;
      if (!mbar_wait_cluster(&tfull[b], (uint32_t)((c >> 1) & 1))) {
        atomicExch(err, 3);
        ok = false;
        break;
      }
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      drain((uint32_t)(b * BNT));
      asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
      __syncwarp();
      if (lane == 0) mbar_arrive_remote(cluster_addr(&tfree[b], 0));
      if (sep && ((c + 1) % corr_mul == 0 || c == nchunk - 1)) {
        const int cc = c / corr_mul, cb = cc & 1;
        if (!mbar_wait_cluster(&cfull[cb], (uint32_t)((cc >> 1) & 1))) {
          atomicExch(err, 6);
          ok = false;
          break;
        }
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        drain((uint32_t)((2 + cb) * BNT));
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        __syncwarp();
        if (lane == 0) mbar_arrive_remote(cluster_addr(&cfree[cb], 0));
      }
    }
    if (ws) {
      float* out = ws + (size_t)blockIdx.z * M * N;
      if (row < M) {
#pragma unroll
        for (int j = 0; j < COLS; ++j) {
          const int col = n0 + cbase + j;
          if (col < N) out[(size_t)col * M + row] = ok ? acc[j] : 0.0f;
        }
      }
    } else if (row < M && ok) {
      double* crow = C + row;
      if (beta == 1.0) {
#pragma unroll
        for (int j = 0; j < COLS; ++j) {
          const int col = n0 + cbase + j;
          if (col < N) atomicAdd(crow + (size_t)col * ldc, alpha * (double)acc[j]);
        }
      } else {
        constexpr int G = (COLS > 64 || EPW > 8) ? 4 : 16;   // loads in flight per group
#pragma unroll
        for (int j0 = 0; j0 < COLS; j0 += G) {
          double old[G];
          if (beta != 0.0) {
#pragma unroll
            for (int j = 0; j < G; ++j) {
              const int col = n0 + cbase + j0 + j;
              old[j] = col < N ? crow[(size_t)col * ldc] : 0.0;
            }
          }
#pragma unroll
          for (int j = 0; j < G; ++j) {
            const int col = n0 + cbase + j0 + j;
            if (col < N)
              crow[(size_t)col * ldc] =
                  alpha * (double)acc[j0 + j] + (beta != 0.0 ? beta * old[j] : 0.0);
          }
        }
      }
    }
  }
  __syncthreads();
  // the pair's MMAs have read both CTAs' shared memory and every arrival has
  // landed before either CTA frees its TMEM or leaves
  cluster_sync_all();
  if (warp == 1) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::2.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                 "r"(tmem_cols)
                 : "memory");
  }
}

}  // namespace tc

// ------------------------------------------------------------------ host
typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*,
                                  const cuuint64_t*, const cuuint64_t*, const cuuint32_t*,
                                  const cuuint32_t*, CUtensorMapInterleave, CUtensorMapSwizzle,
                                  CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

// looked up once; the function-local static's initialisation is thread-safe
// (concurrent steps of several systems)
static EncodeTiledFn encode_fn() {
  static const EncodeTiledFn fn = []() {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    QBX_CUDA(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q));
    QBX_REQUIRE(p && q == cudaDriverEntryPointSuccess, 52, "cuTensorMapEncodeTiled unavailable");
    return (EncodeTiledFn)p;
  }();
  return fn;
}

// K-major matrix of BF16 or TF32 (FP32) elements: rows = k (contiguous, ld
// elements), cols = m; box of one 128-byte row of K by 128 columns, 128-byte
// swizzle.  Columns past `cols` and K past `k` read as zero.
static CUtensorMap kmajor_map(const void* ptr, int k, int cols, int ld, int kind,
                              int box_cols = tc::BM) {
  CUtensorMap map;
  const size_t es = kind == tc::KIND_BF16 ? 2 : 4;
  const cuuint64_t dims[2] = {(cuuint64_t)k, (cuuint64_t)cols};
  const cuuint64_t strides[1] = {(cuuint64_t)ld * es};
  const cuuint32_t box[2] = {(cuuint32_t)tc::bk_of(kind), (cuuint32_t)box_cols};
  const cuuint32_t estr[2] = {1, 1};
  const CUresult r = encode_fn()(
      &map, kind == tc::KIND_BF16 ? CU_TENSOR_MAP_DATA_TYPE_BFLOAT16 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32,
      2, const_cast<void*>(ptr), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
      CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
      CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  QBX_REQUIRE(r == CUDA_SUCCESS, 53, "cuTensorMapEncodeTiled failed: " + std::to_string((int)r));
  return map;
}

// MN-major matrix (M contiguous, ld elements between K rows): boxes of 128
// bytes of M by one K block, 128-byte swizzle (with 32-byte atoms for TF32)
static CUtensorMap mn_map(const void* ptr, int m, int k, int ld, int kind) {
  CUtensorMap map;
  const size_t es = kind == tc::KIND_BF16 ? 2 : 4;
  const cuuint64_t dims[2] = {(cuuint64_t)m, (cuuint64_t)k};
  const cuuint64_t strides[1] = {(cuuint64_t)ld * es};
  const cuuint32_t box[2] = {(cuuint32_t)(128 / es), (cuuint32_t)tc::bk_of(kind)};
  const cuuint32_t estr[2] = {1, 1};
  const CUresult r = encode_fn()(
      &map, kind == tc::KIND_BF16 ? CU_TENSOR_MAP_DATA_TYPE_BFLOAT16 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32,
      2, const_cast<void*>(ptr), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
      kind == tc::KIND_BF16 ? CU_TENSOR_MAP_SWIZZLE_128B : CU_TENSOR_MAP_SWIZZLE_128B_ATOM_32B,
      CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  QBX_REQUIRE(r == CUDA_SUCCESS, 53, "cuTensorMapEncodeTiled failed: " + std::to_string((int)r));
  return map;
}

// out(col * ldc + row) = alpha * sum_s ws(s, col * M + row) + beta * out, in FP64
// (lower: only the tiles the GEMM formed, those that meet the lower triangle)
__global__ void k_reduce_splits2d(const float* __restrict__ ws, int nsplit, int M, int N,
                                  double alpha, double beta, double* __restrict__ out, int ldc,
                                  int lower) {
  const size_t n = (size_t)M * N;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    const size_t col = i / M, row = i - col * M;
    if (lower && (col / tc::BN) * tc::BN >= (row / tc::BM) * tc::BM + tc::BM) continue;
    double s = 0.0;
    for (int z = 0; z < nsplit; z++) s += (double)ws[(size_t)z * n + i];
    double* o = out + col * ldc + row;
    *o = alpha * s + (beta != 0.0 ? beta * *o : 0.0);
  }
}

bool tc_gemm_supported(const Context& ctx, bool ta, bool tb, int m, int n, int k) {
  // transposed-A x plain-B products on whole 128 x 128 tiles, with 16-byte
  // aligned leading dimensions (checked by the caller's padding)
  (void)ctx;
  return ta && !tb && m % tc::BM == 0 && n % tc::BN == 0 && k >= tc::BK;
}

// C (m x n, ld ldc) = alpha * A^T B + beta * C, A (k x m) and B (k x n)
// K-major splits of the given kind.  The K dimension is split across CTAs
// only when the output has too few tiles to fill the GPU.
// amn: A is MN-major (m contiguous, lda between its k rows), CTA pairs on
// 256 x 256 tiles only.
static void tc_gemm_tn(Context& ctx, int kind, int m, int n, int k, double alpha, const void* ahi,
                       const void* alo, int lda, const void* bhi, const void* blo, int ldb,
                       double beta, double* C, int ldc, bool lower = false, bool amn = false) {
  const size_t es = kind == tc::KIND_BF16 ? 2 : 4;
  QBX_REQUIRE(m > 0 && n > 0 && k > 0 && ldc >= m, 54, "bad tcgen05 GEMM shape");
  QBX_REQUIRE((lda * es) % 16 == 0 && (ldb * es) % 16 == 0, 54,
              "leading dimension not 16-byte aligned");
  QBX_REQUIRE(((uintptr_t)ahi | (uintptr_t)alo | (uintptr_t)bhi | (uintptr_t)blo) % 16 == 0, 54,
              "operand not 16-byte aligned");
  QBX_REQUIRE(!amn || ctx.tc_pair == 2, 54, "an MN-major A needs the 256 x 256 CTA-pair kernel");
  const CUtensorMap mah = amn ? mn_map(ahi, m, k, lda, kind) : kmajor_map(ahi, k, m, lda, kind);
  const CUtensorMap mal = amn ? mn_map(alo, m, k, lda, kind) : kmajor_map(alo, k, m, lda, kind);
  const CUtensorMap mbh = kmajor_map(bhi, k, n, ldb, kind);
  const CUtensorMap mbl = kmajor_map(blo, k, n, ldb, kind);
  const int bk = tc::bk_of(kind);
  const int nkb = (k + bk - 1) / bk;
  // tile width: 256 columns for CTA pairs with QBX_TC_PAIR=2, else 128
  const int bnt = ctx.tc_pair == 2 ? 256 : tc::BN;
  const int tm = (m + tc::BM - 1) / tc::BM, tn = (n + bnt - 1) / bnt;
  QBX_REQUIRE(!lower || m == n, 54, "lower-triangle GEMM of a non-square output");
  // tiles formed: with lower, those that meet the lower triangle
  int tiles = tm * tn;
  if (lower) {
    tiles = 0;
    for (int i = 0; i < tm; i++) tiles += std::min(tn, ((i + 1) * tc::BM + bnt - 1) / bnt);
  }
  int sms = 148;
  QBX_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx.device));
  // Split K when the output has few tiles: one CTA per SM runs at a time
  // (its three pipeline stages fill the shared memory), so the CTAs should
  // fill whole waves of sms (a product of fewer than sms/16 tiles gets one
  // wave of short K slices).  Otherwise, of 1..16 splits with K slices of at
  // least 16 blocks, take the one whose waves are fullest, a larger count only for 2 %
  // more (a 64-tile n x n product: 9 splits, 576 CTAs in 3.9 waves, where
  // rounding two CTAs per SM up gave 320 CTAs in 2.2 waves).  The FP32
  // partials are summed in FP64 afterwards.
  int splits = 1;
  if (tiles * 16 < sms) {
    // a small product: one wave of short K slices
    splits = std::max(1, std::min(nkb, (sms + tiles - 1) / tiles));
  } else if (tiles < 4 * sms) {
    double best = -1.0;
    for (int sp = 1; sp <= 16 && (nkb + sp - 1) / sp >= 16; sp++) {
      const long work = (long)tiles * sp;
      const long waves = (work + sms - 1) / sms;
      const double eff = (double)work / (double)(waves * sms);
      if (eff > best + 0.02) {
        best = eff;
        splits = sp;
      }
    }
  }
  const int kbps = (nkb + splits - 1) / splits;
  splits = (nkb + kbps - 1) / kbps;
  if (splits > 1) {
    const size_t need = (size_t)splits * m * n;
    if (need > ctx.tc_ws_elems) {
      // a captured step replays fixed pointers: the workspace is sized by an
      // eager run of the same step before its capture
      QBX_REQUIRE(!ctx.capturing, 56, "split-K workspace growth while capturing a step");
      if (ctx.d_tc_ws) cudaFree(ctx.d_tc_ws);
      ctx.d_tc_ws = nullptr;
      ctx.tc_ws_elems = 0;
      QBX_CUDA(cudaMalloc(&ctx.d_tc_ws, need * sizeof(float)));
      ctx.tc_ws_elems = need;
    }
  }
  int* err = ctx.d_status + ST_TC_ERR;   // wait-timeout flag, sticky
  const int chunk = std::max(1, ctx.tc_chunk), corr_mul = std::max(0, ctx.tc_corr_mul);
  float* ws = splits > 1 ? (float*)ctx.d_tc_ws : nullptr;
  if (ctx.tc_pair) {
    // CTA pairs: B in half tiles of bnt / 2 columns, M tiles padded to an
    // even count; 256-column tiles keep the correction terms in the hi*hi
    // chain and use eight epilogue warps
    const CUtensorMap mbh2 = kmajor_map(bhi, k, n, ldb, kind, bnt / 2);
    const CUtensorMap mbl2 = kmajor_map(blo, k, n, ldb, kind, bnt / 2);
    const int cm = bnt == 256 ? 0 : corr_mul;
    const int tm2 = (tm + 1) & ~1;
    QBX_REQUIRE(splits > 1 ? tn <= 65535 : tm2 / 2 <= 65535, 54, "too many tiles for the grid");
    const dim3 grid2 = splits > 1 ? dim3(tm2, tn, splits) : dim3(2 * tn, tm2 / 2, 1);
    auto launch2 = [&](auto kern, int epw, int smem) {
      allow_smem(kern, smem);
      cudaLaunchConfig_t cfg = {};
      cfg.gridDim = grid2;
      cfg.blockDim = dim3(tc::threads_of(epw));
      cfg.dynamicSmemBytes = smem;
      cfg.stream = ctx.stream;
      cudaLaunchAttribute at[1];
      at[0].id = cudaLaunchAttributeClusterDimension;
      at[0].val.clusterDim.x = 2;   // a cta_group::2 pair is a cluster along x
      at[0].val.clusterDim.y = 1;
      at[0].val.clusterDim.z = 1;
      cfg.attrs = at;
      cfg.numAttrs = 1;
      QBX_CUDA(cudaLaunchKernelEx(&cfg, kern, mah, mal, mbh2, mbl2, m, n, nkb, kbps, ws, C, ldc,
                                  alpha, beta, err, lower ? 1 : 0, chunk, cm));
    };
    constexpr int S128 = tc::PairCfg<128>::SMEM_BYTES, S256 = tc::PairCfg<256>::SMEM_BYTES;
    const bool e16 = ctx.tc_pair_epw == 16;
    if (kind == tc::KIND_BF16) {
      if (amn && e16) launch2(tc::k_tc_pair_gemm<tc::KIND_BF16, 16, 256, true>, 16, S256);
      else if (amn) launch2(tc::k_tc_pair_gemm<tc::KIND_BF16, 8, 256, true>, 8, S256);
      else if (bnt == 256 && e16) launch2(tc::k_tc_pair_gemm<tc::KIND_BF16, 16, 256, false>, 16, S256);
      else if (bnt == 256) launch2(tc::k_tc_pair_gemm<tc::KIND_BF16, 8, 256, false>, 8, S256);
      else if (ctx.tc_epw == 8) launch2(tc::k_tc_pair_gemm<tc::KIND_BF16, 8, 128, false>, 8, S128);
      else launch2(tc::k_tc_pair_gemm<tc::KIND_BF16, 4, 128, false>, 4, S128);
    } else {
      if (amn && e16) launch2(tc::k_tc_pair_gemm<tc::KIND_TF32, 16, 256, true>, 16, S256);
      else if (amn) launch2(tc::k_tc_pair_gemm<tc::KIND_TF32, 8, 256, true>, 8, S256);
      else if (bnt == 256 && e16) launch2(tc::k_tc_pair_gemm<tc::KIND_TF32, 16, 256, false>, 16, S256);
      else if (bnt == 256) launch2(tc::k_tc_pair_gemm<tc::KIND_TF32, 8, 256, false>, 8, S256);
      else if (ctx.tc_epw == 8) launch2(tc::k_tc_pair_gemm<tc::KIND_TF32, 8, 128, false>, 8, S128);
      else launch2(tc::k_tc_pair_gemm<tc::KIND_TF32, 4, 128, false>, 4, S128);
    }
  } else {
    QBX_REQUIRE(splits > 1 ? tn <= 65535 : tm <= 65535, 54, "too many tiles for the grid");
    const dim3 grid = splits > 1 ? dim3(tm, tn, splits) : dim3(tn, tm, 1);
    auto launch = [&](auto kern, int epw) {
      allow_smem(kern, tc::SMEM_BYTES);
      kern<<<grid, tc::threads_of(epw), tc::SMEM_BYTES, ctx.stream>>>(
          mah, mal, mbh, mbl, m, n, nkb, kbps, ws, C, ldc, alpha, beta, err, lower ? 1 : 0,
          chunk, corr_mul);
    };
    if (kind == tc::KIND_BF16) {
      if (ctx.tc_epw == 8) launch(tc::k_tc_split_gemm<tc::KIND_BF16, 8>, 8);
      else launch(tc::k_tc_split_gemm<tc::KIND_BF16, 4>, 4);
    } else {
      if (ctx.tc_epw == 8) launch(tc::k_tc_split_gemm<tc::KIND_TF32, 8>, 8);
      else launch(tc::k_tc_split_gemm<tc::KIND_TF32, 4>, 4);
    }
  }
  QBX_LAUNCHED(ctx);
  if (splits > 1) {
    const size_t nn = (size_t)m * n;
    const int nb = (int)std::min<size_t>((nn + 255) / 256, (size_t)sms * 16);
    k_reduce_splits2d<<<nb, 256, 0, ctx.stream>>>((const float*)ctx.d_tc_ws, splits, m, n, alpha,
                                                  beta, C, ldc, lower ? 1 : 0);
    QBX_LAUNCHED(ctx);
  }
}

void tc_split_gemm(Context& ctx, bool ta, bool tb, int m, int n, int k, double alpha,
                   const void* ahi, const void* alo, int lda, const void* bhi, const void* blo,
                   int ldb, double beta, double* C, bool lower) {
  QBX_REQUIRE(tc_gemm_supported(ctx, ta, tb, m, n, k), 54, "shape not supported by tcgen05 GEMM");
  tc_gemm_tn(ctx, tc::KIND_BF16, m, n, k, alpha, ahi, alo, lda, bhi, blo, ldb, beta, C, m, lower);
}

void tc_gemm_kind_tn(Context& ctx, int kind, int m, int n, int k, double alpha, const void* ahi,
                     const void* alo, int lda, const void* bhi, const void* blo, int ldb,
                     double beta, double* C, int ldc) {
  tc_gemm_tn(ctx, kind == TALL_TF32 ? tc::KIND_TF32 : tc::KIND_BF16, m, n, k, alpha, ahi, alo, lda,
             bhi, blo, ldb, beta, C, ldc);
}

void tc_gemm_kind_nn_mn(Context& ctx, int kind, int m, int n, int k, double alpha, const void* ahi,
                        const void* alo, int lda, const void* bhi, const void* blo, int ldb,
                        double beta, double* C, int ldc) {
  tc_gemm_tn(ctx, kind == TALL_TF32 ? tc::KIND_TF32 : tc::KIND_BF16, m, n, k, alpha, ahi, alo, lda,
             bhi, blo, ldb, beta, C, ldc, false, true);
}

void tc_tf32_gemm_tn(Context& ctx, int m, int n, int k, double alpha, const float* ahi,
                     const float* alo, int lda, const float* bhi, const float* blo, int ldb,
                     double beta, double* C, int ldc) {
  tc_gemm_tn(ctx, tc::KIND_TF32, m, n, k, alpha, ahi, alo, lda, bhi, blo, ldb, beta, C, ldc);
}

int tc_check_error(Context& ctx) {
  if (!ctx.d_status) return 0;
  int e = 0;
  QBX_CUDA(cudaMemcpyAsync(&e, ctx.d_status + ST_TC_ERR, sizeof(int), cudaMemcpyDeviceToHost,
                           ctx.stream));
  QBX_CUDA(cudaStreamSynchronize(ctx.stream));
  return e;
}

}  // namespace qbx
