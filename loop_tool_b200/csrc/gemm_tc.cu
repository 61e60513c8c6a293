// Family (c) on the 5th-generation tensor cores: tcgen05.mma (kind::f16,
// BF16 inputs, FP32 accumulation in TMEM) fed by TMA through an mbarrier
// pipeline, persistent over a table of problems (one problem for a single
// contraction, hundreds for a batch of uneven matmuls in one launch).
//
// Operands arrive as dense K-major BF16 matrices A'[M, Kp], B'[N, Kp] made by
// the operand packer (k_pack_one / k_pack_grouped) from the contraction's
// separable FP32 operand description, so the same kernel runs matmul,
// batched matmul and gathered operands.  A convolution's input can instead
// be an image operand: packed once as a zero-padded NHWC BF16 image
// (k_pack_image, or k_pack_conv with the weights in the same launch) and
// loaded as 4-D TMA boxes per output image row (implicit GEMM, no im2col
// matrix).  The split-BF16 modes pack A' = [Ah | Al | Ah
// (| Al)], B' = [Bh | Bh | Bl (| Bl)] along K, so one BF16 GEMM accumulates
// Ah*Bh + Al*Bh + Ah*Bl (+ Al*Bl); the six-product mode splits each value
// into three pieces (hi + lo + lo2 == x) and adds Al*Bl + Al2*Bh + Ah*Bl2.
//
// Chunked accumulation.  The tensor core's FP32 accumulation truncates, so
// its error grows linearly with the number of K steps summed into one TMEM
// accumulator (measured: ~1.9e-5 relative at K = 16384 with BF16-exact
// inputs).  The K loop is therefore cut into chunks, each accumulated from
// zero in one of two TMEM buffers (LtbTcProblem::chunk_blocks, main_blocks,
// rest_blocks; chunk_len): the whole K for plain BF16, whose input rounding
// outweighs the truncation by far; for the split modes, short chunks on the
// main segment (Ah.Bh: 512 K, 128 K in the six-product mode) and long ones
// (4096 K, 512 K) on the correction segments, whose products are 2^-8 of
// the main ones.  Drain warps read a finished chunk back (16 columns per
// tcgen05.ld) and add it into FP32 registers with round-to-nearest adds
// while the tensor core fills the other buffer.
//
// Tile forms (a tuned schedule): 128 x 256 or 128 x 128 output tiles, one CTA
// per SM (4- or 6-stage ring), or two 128 x 128 CTAs per SM (3-stage rings);
// epilogue by per-thread row stores (32-byte sector stores where aligned) or
// through a 32 x 32 shared-memory transpose into whole-row stores.  Halo
// image tiles (single-segment convolutions, N <= 128): the weights stay
// resident in shared memory and one 4-D box per (tile, channel block) -- the
// tile's padded image rows and the kh - 1 rows below them -- serves every
// (kh, kw) shift, read in place.
//
// Roles (320 threads per CTA):
//   warp 0 lane 0 : TMA producer                  warp 0 : TMEM alloc/free
//   warp 1 lane 0 : MMA issuer (4 x K=16 tcgen05.mma per 64-wide k block)
//   warps 2..9    : drain + epilogue; warp w reads TMEM lanes 32*(w%4)..+31
//                   and half (w-2)/4 of the tile's columns
// Every wait is bounded: on timeout a flag is raised for the host
// (LTB_ERR_TIMEOUT) and the CTA winds down without hanging.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cudaTypedefs.h>

#include <map>
#include <mutex>
#include <tuple>

#include "async.cuh"
#include "kernels.h"
#include "tc_api.h"

namespace {

constexpr int BM = 128, BK = 64;
constexpr int NT = 320;
constexpr int kChunkBlocks = 8;  // default: 8 x 64 = 512 K elements per accumulator
constexpr int A_BYTES = BM * BK * 2;
// epilogue: each drain warp transposes 32 x 32 blocks through a padded
// shared buffer so global stores are whole 128-byte row segments (outputs
// that TMA cannot store)
constexpr int kEpiPitch = 33;

// Tile shapes: BM x BN output tiles, BN = 256 (4-stage ring of 48 KB) or
// BN = 128 (6-stage ring of 32 KB; narrow outputs and small problems).
// CTAS = 2: two CTAs share an SM (BN = 128, 3-stage rings, row-store
// epilogue), each hiding the other's load latency and epilogue.
template <int BN_, int CTAS = 1>
struct Tile {
  static constexpr int B_BYTES = BN_ * BK * 2;
  static constexpr int STAGE_BYTES = A_BYTES + B_BYTES;
  static constexpr int STAGES = CTAS == 2 ? 3 : BN_ == 256 ? 4 : 6;
  static constexpr uint32_t TMEM_COLS = 2 * BN_;  // two accumulator buffers
  static constexpr int HALF = BN_ / 2;            // columns per drain thread
  // kind::f16 instruction descriptor: FP32 accumulator, BF16 A and B, both
  // K-major, M = 128, N = BN
  static constexpr uint32_t IDESC = (1u << 4) | (1u << 7) | (1u << 10) |
                                    ((uint32_t)(BN_ >> 3) << 17) | ((uint32_t)(BM >> 4) << 24);
  // dynamic: ring + alignment slack + barriers (the epilogue buffers are
  // static shared memory, kEpiBytes more per CTA)
  static constexpr size_t SMEM = (size_t)STAGES * STAGE_BYTES + 1024 + 256;
  // launches with TMA-stored outputs and no transposed-epilogue buffer:
  // 32 KB of staging 1024 bytes after the ring (past its barriers)
  static constexpr size_t SMEM_TMA = (size_t)STAGES * STAGE_BYTES + 1024 + 1024 + 8 * 4096;
};
__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap* map, uint32_t bar,
                                            int x, int y) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3}], [%4];" ::"r"(dst),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(bar)
      : "memory");
}

// 4-D box (image operands: channels, columns, row, image); coordinates
// outside the image read as zeros.
__device__ __forceinline__ void tma_load_4d(uint32_t dst, const CUtensorMap* map, uint32_t bar,
                                            int x, int y, int z, int w) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3, %4, %5}], [%6];" ::"r"(dst),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(w), "r"(bar)
      : "memory");
}

// 2-D box shared -> global (the output tile's 32 x 32 FP32 blocks), in this
// thread's bulk async-group; the parts of the box outside the tensor are
// not written.
__device__ __forceinline__ void tma_store_2d(const CUtensorMap* map, uint32_t src, int x, int y) {
  asm volatile("cp.async.bulk.tensor.2d.global.shared::cta.bulk_group [%0, {%1, %2}], [%3];" ::"l"(
                   reinterpret_cast<uint64_t>(map)),
               "r"(x), "r"(y), "r"(src)
               : "memory");
}
__device__ __forceinline__ void bulk_commit() {
  asm volatile("cp.async.bulk.commit_group;" ::: "memory");
}
// this thread's bulk stores have read their shared-memory sources
__device__ __forceinline__ void bulk_wait_read() {
  asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");
}
// this thread's bulk stores are complete
__device__ __forceinline__ void bulk_wait() {
  asm volatile("cp.async.bulk.wait_group 0;" ::: "memory");
}
// generic-proxy shared-memory writes made visible to the TMA (async proxy)
__device__ __forceinline__ void fence_async_shared() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// Output row of tile row tr (0..127) of m-tile m0 / BM, and whether the row
// exists: plain operands map tile rows to rows m0 + tr; image operands to
// image row tr / img_slot, column tr % img_slot of the tile's image rows.
__device__ __forceinline__ bool tile_row(const LtbTcProblem& p, int m0, int tr, int* row) {
  if (!p.img) {
    *row = m0 + tr;
    return *row < p.M;
  }
  const int mt = m0 / BM, n_img = mt / p.img_hgroups;
  const int ho0 = (mt - n_img * p.img_hgroups) * p.img_rows;
  const int i = tr / p.img_slot, w = tr - i * p.img_slot;
  const bool ok = i < p.img_rows && w < p.img_wo && ho0 + i < p.img_ho;
  *row = ok ? (n_img * p.img_ho + ho0 + i) * p.img_wo + w : 0;
  return ok;
}

// K-major, 128-byte-swizzled canonical layout: 8-row x 128-byte atoms
// (1024 B) stacked along M/N, LBO unused (1), SBO = 1024 B, version 1.
__device__ __forceinline__ uint64_t sw128_desc(uint32_t addr) {
  return (uint64_t)((addr >> 4) & 0x3FFF) | (uint64_t)1 << 16 | (uint64_t)(1024 >> 4) << 32 |
         (uint64_t)1 << 46 | (uint64_t)2 << 61;
}

// An operand may also start at any 128-byte row inside a 1024-byte swizzle
// atom (a halo tile read from row kw): the swizzle follows the absolute
// shared-memory address bits, as the TMA wrote it, so the matrix base offset
// field stays 0 (measured: setting it to the row phase gives wrong sums).

__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t idesc,
                                         uint32_t accumulate) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
      " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem_d),
      "l"(a), "l"(b), "r"(idesc), "r"(accumulate));
}

__device__ __forceinline__ void mma_commit(uint32_t bar) {
  asm volatile(
      "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
      : "memory");
}

// 16 consecutive 32-bit columns of the warp's 32 TMEM lanes (one per thread)
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t* r) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, "
      "%11, %12, %13, %14, %15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
        "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
}

// 32 bytes (8 floats) to a 32-byte aligned global address: one whole L2
// sector per thread and instruction.
__device__ __forceinline__ void st_global_v8(float* dst, const float* v) {
  asm volatile("st.global.v8.f32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8};" ::"l"(dst), "f"(v[0]),
               "f"(v[1]), "f"(v[2]), "f"(v[3]), "f"(v[4]), "f"(v[5]), "f"(v[6]), "f"(v[7])
               : "memory");
}

__device__ __forceinline__ void tmem_wait_ld() {
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// Tile index -> (problem, m0, n0).  Tiles of a problem run M-fastest so
// consecutive CTAs share the B tile in L2.
__device__ __forceinline__ int find_problem(const LtbTcProblem* __restrict__ P, int np,
                                            int64_t t) {
  int lo = 0, hi = np - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (P[mid].tile_start <= t) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

// Length of the accumulation chunk that starts at k block c0 of nk:
// chunk_blocks (0: kChunkBlocks) within the first main_blocks, rest_blocks
// past them when rest_blocks is set (the main part's last chunk ends with
// it).  The MMA issuer and the drain warps cut K the same way.
__device__ __forceinline__ int chunk_len(const LtbTcProblem& p, int c0, int nk) {
  int len = p.chunk_blocks > 0 ? p.chunk_blocks : kChunkBlocks;
  if (p.rest_blocks > 0) {
    if (c0 >= p.main_blocks) len = p.rest_blocks;
    else if (c0 + len > p.main_blocks) len = p.main_blocks - c0;
  }
  return c0 + len < nk ? len : nk - c0;
}

// The i-th tile of work unit u (a CTA, or a cluster of two CTAs): from the
// unit's span of a host-built order when there is one (a batch's
// longest-first assignment of uneven tiles to units), else tile u + i *
// step.  False past the unit's last tile.
__device__ __forceinline__ bool tile_at(const int* __restrict__ order,
                                        const int* __restrict__ ostart, int64_t u, int64_t step,
                                        int64_t total, int64_t i, int64_t* t) {
  if (order) {
    const int64_t b = ostart[u];
    if (i >= ostart[u + 1] - b) return false;
    *t = order[b + i];
    return true;
  }
  *t = u + i * step;
  return *t < total;
}

// Grouped raster: tiles advance along M in groups of group_m row blocks (a
// per-problem schedule, 16 by default), so the ~148 tiles in flight cover a
// compact block region whose A and B panels stay resident in L2.
template <int BN>
__device__ __forceinline__ void tile_coords(const LtbTcProblem& p, int64_t lt, int* m0, int* n0) {
  const int gmax = p.group_m > 0 ? p.group_m : 16;
  const int64_t per_group = (int64_t)gmax * p.tiles_n;
  const int g = (int)(lt / per_group);
  const int idx = (int)(lt - (int64_t)g * per_group);
  const int gm = p.tiles_m - g * gmax < gmax ? p.tiles_m - g * gmax : gmax;
  *m0 = (g * gmax + idx % gm) * BM;
  *n0 = (idx / gm) * BN;
}

// Writes a drain warp's share of a finished tile: rows m0 + 32*quad .. +31
// (row m0 + 32*quad + lane in this thread's run[]) and HALF columns from
// cbase.  Three forms: TMA stores of 32 x 32 blocks staged 128-byte
// swizzled in the warp's 4 KB of shared memory (kTma, outputs whose rows are
// one progression of 16-byte multiples: LtbTcProblem::c_tma), whole-row
// stores through a padded 32 x 32 transpose (kTE, unit columns), or each
// thread's own row (32-byte sector stores where aligned, else float4 or
// scalar, through the column table when columns are not unit).
template <int HALF, bool kTma, bool kTE>
__device__ __forceinline__ void write_tile(const LtbTcProblem& p, const CUtensorMap* mc,
                                           float* c_override, const float (&run)[HALF],
                                           float* epi, int ew, int m0, int cbase, bool rvalid,
                                           int64_t rbase) {
  const int lane = threadIdx.x & 31, quad = threadIdx.x >> 5 & 3;
  float* cb = c_override ? c_override : p.c;
  if (kTma && p.c_tma && !c_override) {
    // 16-byte chunk q of row r at chunk q ^ (r % 8): conflict-free float4
    // writes; the stores run on while the warp drains the next tile, and the
    // buffer is rewritten once the previous store has read it
    float* stage = epi + ew * 1024;
    if (m0 + 32 * quad >= p.M) return;  // no row of this warp's blocks exists
#pragma unroll
    for (int c = 0; c < HALF; c += 32) {
      if (cbase + c >= p.N) break;  // nor any column from here on
      if (lane == 0) bulk_wait_read();
      __syncwarp();
#pragma unroll
      for (int q = 0; q < 8; ++q)
        *reinterpret_cast<float4*>(stage + lane * 32 + ((q ^ (lane & 7)) << 2)) =
            make_float4(run[c + 4 * q], run[c + 4 * q + 1], run[c + 4 * q + 2],
                        run[c + 4 * q + 3]);
      fence_async_shared();
      __syncwarp();
      if (lane == 0) {
        tma_store_2d(mc, smem_u32(stage), cbase + c, m0 + 32 * quad);
        bulk_commit();
      }
    }
  } else if (kTE && p.unit_cols) {
    float* stage = epi + ew * (32 * kEpiPitch);
    const int64_t rb = rbase;
#pragma unroll
    for (int c = 0; c < HALF; c += 32) {
      __syncwarp();
#pragma unroll
      for (int j = 0; j < 32; ++j) stage[lane * kEpiPitch + j] = run[c + j];
      __syncwarp();
      const int col = cbase + c + lane;
      const bool cok = col < p.N;
#pragma unroll 8
      for (int i = 0; i < 32; ++i) {  // row i of the block: 32 consecutive columns
        const int64_t rbi = __shfl_sync(0xffffffffu, rb, i);
        const int vi = __shfl_sync(0xffffffffu, (int)rvalid, i);
        if (vi && cok) cb[rbi + col] = stage[i * kEpiPitch + lane];
      }
    }
  } else if (rvalid) {  // this thread's row: 32-byte (whole sector) stores where aligned
    float* dst = cb + rbase;
#pragma unroll
    for (int c = 0; c < HALF; c += 8) {
      const int j = cbase + c;
      if (p.unit_cols && j + 8 <= p.N && (reinterpret_cast<uintptr_t>(dst + j) & 31) == 0) {
        st_global_v8(dst + j, &run[c]);
        continue;
      }
#pragma unroll
      for (int h = 0; h < 8; h += 4) {
        const int jh = j + h;
        if (p.unit_cols && jh + 4 <= p.N && ((rbase + jh) & 3) == 0) {
          *reinterpret_cast<float4*>(dst + jh) =
              make_float4(run[c + h], run[c + h + 1], run[c + h + 2], run[c + h + 3]);
        } else {
#pragma unroll
          for (int e = 0; e < 4; ++e)
            if (jh + e < p.N) dst[p.unit_cols ? jh + e : p.ccol[jh + e]] = run[c + h + e];
        }
      }
    }
  }
}

// 10 warps per CTA: the SM's four register partitions (16K each) hold up to
// three warps each, so at most 168 registers per thread.
// Halo tiles: resident B' (every 64-wide k block of the 128-row panel) and
// a ring of at most kMaxHaloStages halo slots, within the 227 KB a CTA may
// use.
constexpr int kMaxHaloStages = 8;
constexpr int kMaxHaloKb = 16;  // resident B' k blocks (one mbarrier each)
constexpr size_t kHaloSmemMax = 227 * 1024;
constexpr size_t kHaloBBytes = (size_t)128 * BK * 2;
// barriers: full/empty per ring slot, one per resident k block, 2 + 2 chunk
// barriers, the TMEM address word
constexpr size_t kHaloBarBytes = (2 * kMaxHaloStages + kMaxHaloKb + 4) * 8 + 8;

template <int BN, bool kTransposeEpi, int CTAS, bool kHalo = false>
__global__ void __launch_bounds__(NT, CTAS)
    k_gemm_tc(const LtbTcProblem* __restrict__ probs, int nprob, int64_t total_tiles,
              float* c_override, int* err, const int* __restrict__ order,
              const int* __restrict__ ostart, const __grid_constant__ LtbTcProblem single,
              const __grid_constant__ CUtensorMap single_a,
              const __grid_constant__ CUtensorMap single_b,
              const __grid_constant__ CUtensorMap single_a2,
              const __grid_constant__ CUtensorMap single_a3,
              const __grid_constant__ CUtensorMap single_c) {
  // probs == nullptr: one problem passed by value with its tensor maps as
  // kernel parameters (encoded at launch over per-run scratch)
  using T = Tile<BN, CTAS>;
  constexpr int STAGES = T::STAGES, STAGE_BYTES = T::STAGE_BYTES;
  extern __shared__ __align__(1024) uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>(
      (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  // ring of STAGES slots, or (halo tiles) resident B' then the halo ring
  int nst = STAGES;
  uint32_t slot_bytes = STAGE_BYTES;
  uint8_t* ring = smem;
  uint8_t* bres = smem;  // halo tiles: B' k block kb at bres + kb * B_BYTES
  int kbt = 0;
  if constexpr (kHalo) {
    kbt = (int)(single.Kp / BK);
    ring = smem + (size_t)kbt * T::B_BYTES;
    nst = single.img_stages;
    slot_bytes = (uint32_t)single.img_slot_bytes;
  }
  uint64_t* full = reinterpret_cast<uint64_t*>(ring + (size_t)nst * slot_bytes);
  uint64_t* empty = full + nst;
  uint64_t* b_full = empty + nst;            // halo tiles: [kbt] resident B' k block loaded
  uint64_t* chunk_full = b_full + (kHalo ? kbt : 1);  // [2] MMA -> drain
  uint64_t* chunk_empty = chunk_full + 2;    // [2] drain -> MMA
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(chunk_empty + 2);
  // drain warps' staging, one region per warp: the transposed form's 32 x
  // 32 transposes (padded pitch), and the 4 KB swizzled blocks of the
  // TMA-store epilogue in the same buffer, or else in 32 KB of dynamic
  // shared memory after the ring's barriers, present only in launches with
  // TMA-stored outputs (SMEM_TMA): image operands keep the L1 capacity
  constexpr bool kTmaEpi = CTAS == 1 && !kHalo;
  constexpr int kEpiFloats = kTransposeEpi ? 8 * 32 * kEpiPitch : 1;
  __shared__ __align__(1024) float epi[kEpiFloats];
  float* tma_stage =
      kTransposeEpi ? epi : reinterpret_cast<float*>(smem + (size_t)STAGES * STAGE_BYTES + 1024);
  static_assert(kHalo || T::SMEM + kEpiFloats * 4 <= 227 * 1024, "shared memory per CTA");
  static_assert(T::SMEM_TMA <= 227 * 1024, "shared memory per CTA");

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

  if (threadIdx.x == 0) {
    for (int s = 0; s < nst; ++s) {
      mbar_init(smem_u32(&full[s]), 1);
      mbar_init(smem_u32(&empty[s]), 1);
    }
    for (int kb = 0; kb < (kHalo ? kbt : 1); ++kb) mbar_init(smem_u32(&b_full[kb]), 1);
    for (int b = 0; b < 2; ++b) {
      mbar_init(smem_u32(&chunk_full[b]), 1);
      mbar_init(smem_u32(&chunk_empty[b]), 8 * 32);  // every drain thread
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(tmem_slot)),
                 "r"(T::TMEM_COLS));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tmem_slot;

  if (kHalo && warp == 0 && lane == 0) {
    // ------------------------------------------------- producer (halo tiles)
    // one box per (tile, channel block): the tile's img_rows image rows and
    // the kh - 1 halo rows below them, every padded column; all kh x kw
    // shifts of the tile are read from it in place
    const LtbTcProblem& p = single;
    const uint32_t box_bytes = (uint32_t)((p.img_rows + p.img_kh - 1) * p.img_slot * 128);
    bool first = true;  // the first tile also loads the resident B' blocks, in first-use order
    uint32_t g = 0;  // stages issued
    bool alive = true;
    for (int64_t t = blockIdx.x; t < total_tiles && alive; t += gridDim.x) {
      int m0, n0;
      tile_coords<BN>(p, t, &m0, &n0);
      const int mt = m0 / BM, n_img = mt / p.img_hgroups;
      const int ho0 = (mt - n_img * p.img_hgroups) * p.img_rows;
      for (int cb = 0; cb < p.img_cblocks; ++cb, ++g) {
        const int s = (int)(g % (uint32_t)nst);
        if (!mbar_wait(smem_u32(&empty[s]), ((g / (uint32_t)nst) & 1u) ^ 1u, err)) {
          alive = false;
          break;
        }
        if (first)
          for (int kh = 0; kh < p.img_kh; ++kh)
            for (int kw = 0; kw < p.img_kw; ++kw) {
              const int kb = (kh * p.img_kw + kw) * p.img_cblocks + cb;
              const uint32_t bb = smem_u32(&b_full[kb]);
              mbar_expect_tx(bb, (uint32_t)T::B_BYTES);
              tma_load_2d(smem_u32(bres + (size_t)kb * T::B_BYTES), &single_b, bb, kb * BK, 0);
            }
        const uint32_t fb = smem_u32(&full[s]);
        mbar_expect_tx(fb, box_bytes);
        tma_load_4d(smem_u32(ring + (size_t)s * slot_bytes), &single_a, fb, cb * 64, 0, ho0,
                    n_img);
      }
      first = false;
    }
    // the last round of each ring slot and the resident B' blocks loaded
    // (those of the first tile's first g channel blocks) have landed
    // before the CTA winds down
    for (uint32_t i = g > (uint32_t)nst ? g - nst : 0; i < g; ++i)
      mbar_drain(smem_u32(&full[i % nst]), (i / nst) & 1u);
    for (int kb = 0; kb < kbt; ++kb)
      if ((uint32_t)(kb % p.img_cblocks) < g) mbar_drain(smem_u32(&b_full[kb]), 0u);
  } else if (kHalo && warp == 1 && lane == 0) {
    // ----------------------------------------------- MMA issuer (halo tiles)
    const LtbTcProblem& p = single;
    uint32_t g = 0, q = 0;  // stages consumed, chunks produced
    bool alive = true;
    bool first = true;  // B' blocks are waited for on first use
    const int nkb = kbt;
    // halo problems keep the default chunk (a compile-time divisor: this
    // single issuing thread is on the MMA's critical path)
    constexpr int cbk = kChunkBlocks;
    // the problem's fields in registers, and the operand descriptors of the
    // (kh, kw) shifts stepped by constants (16-byte units: one padded image
    // row per kh, one pixel per kw, the channel blocks' weight blocks per
    // shift): few instructions between this thread's MMAs
    const int khn = p.img_kh, kwn = p.img_kw, ncb = p.img_cblocks;
    const uint64_t a_kh = (uint64_t)p.img_slot * 8u;
    const uint64_t b_blk = (uint64_t)(T::B_BYTES >> 4), b_shift = (uint64_t)ncb * b_blk;
    const uint64_t b0 = sw128_desc(smem_u32(bres));
    for (int64_t t = blockIdx.x; t < total_tiles && alive; t += gridDim.x) {
      int issued = 0, buf = 0;
      uint32_t acc = tmem;
      for (int cb = 0; cb < ncb && alive; ++cb, ++g) {
        const int s = (int)(g % (uint32_t)nst);
        if (!mbar_wait(smem_u32(&full[s]), (g / (uint32_t)nst) & 1u, err)) {
          alive = false;
          break;
        }
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        uint64_t arow = sw128_desc(smem_u32(ring + (size_t)s * slot_bytes));
        uint64_t bd = b0 + (uint64_t)cb * b_blk;
        int kb = cb;  // (kh * kw_n + kw) * cblocks + cb
        for (int kh = 0; kh < khn && alive; ++kh, arow += a_kh)
          for (int kw = 0; kw < kwn; ++kw, bd += b_shift, kb += ncb) {
            if (issued % cbk == 0) {  // a new accumulation chunk
              buf = (int)(q & 1u);
              if (!mbar_wait(smem_u32(&chunk_empty[buf]), ((q >> 1) & 1u) ^ 1u, err)) {
                alive = false;
                break;
              }
              asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
              acc = tmem + (uint32_t)(buf * BN);
            }
            if (first && !mbar_wait(smem_u32(&b_full[kb]), 0u, err)) {
              alive = false;
              break;
            }
            // shift (kh, kw): tile row i * wp + w reads box row
            // (i + kh) * wp + (w + kw), 128 bytes a row
            const uint64_t ad = arow + 8u * (uint64_t)kw;
#pragma unroll
            for (int kk = 0; kk < BK / 16; ++kk)
              mma_bf16(acc, ad + 2 * kk, bd + 2 * kk, T::IDESC,
                       (issued % cbk != 0) || (kk != 0));
            ++issued;
            if (issued % cbk == 0 || issued == nkb) {
              mma_commit(smem_u32(&chunk_full[buf]));  // chunk complete in TMEM
              ++q;
            }
          }
        mma_commit(smem_u32(&empty[s]));  // slot reusable once these finish
      }
      first = false;
    }
  } else if (!kHalo && warp == 0 && lane == 0) {
    // ------------------------------------------------------------ producer
    uint32_t g = 0;  // k blocks issued by this CTA so far
    bool alive = true;
    for (int64_t i = 0, t;
         alive && tile_at(order, ostart, blockIdx.x, gridDim.x, total_tiles, i, &t); ++i) {
      const LtbTcProblem& p = probs ? probs[find_problem(probs, nprob, t)] : single;
      const CUtensorMap* ma =
          probs ? static_cast<const CUtensorMap*>(p.map_a) : &single_a;
      const CUtensorMap* mb =
          probs ? static_cast<const CUtensorMap*>(p.map_b) : &single_b;
      const CUtensorMap* ma2 =
          probs ? static_cast<const CUtensorMap*>(p.map_a2) : &single_a2;
      const CUtensorMap* ma3 =
          probs ? static_cast<const CUtensorMap*>(p.map_a3) : &single_a3;
      int m0, n0;
      tile_coords<BN>(p, t - p.tile_start, &m0, &n0);
      const int nk = (int)((p.Kp + BK - 1) / BK);
      // image operands: this tile's image and first output image row
      const int mt = m0 / BM;
      const int n_img = p.img ? mt / p.img_hgroups : 0;
      const int ho0 = p.img ? (mt - n_img * p.img_hgroups) * p.img_rows : 0;
      const int kseg = p.img ? p.img_kh * p.img_kw * p.img_cblocks : 1;
      for (int kb = 0; kb < nk; ++kb, ++g) {
        const int s = g % STAGES;
        const uint32_t ph = (g / STAGES) & 1u;
        if (!mbar_wait(smem_u32(&empty[s]), ph ^ 1u, err)) {
          alive = false;
          break;
        }
        const uint32_t fb = smem_u32(&full[s]);
        uint8_t* sa = smem + s * STAGE_BYTES;
        if (p.img) {
          // k-block -> (segment, kh, kw, channel block); one box per image row
          const int seg = kb / kseg, r = kb - seg * kseg;
          const int cb = r % p.img_cblocks, r2 = r / p.img_cblocks;
          const int kw = r2 % p.img_kw, kh = r2 / p.img_kw;
          const CUtensorMap* m = (p.img_a_mask >> (8 + seg)) & 1 ? ma3
                                 : (p.img_a_mask >> seg) & 1    ? ma
                                                                : ma2;
          mbar_expect_tx(fb, (uint32_t)(p.img_rows * p.img_wo * 128 + T::B_BYTES));
          for (int i = 0; i < p.img_rows; ++i)
            tma_load_4d(smem_u32(sa + i * p.img_slot * 128), m, fb, cb * 64, kw, ho0 + i + kh,
                        n_img);
        } else {
          mbar_expect_tx(fb, STAGE_BYTES);
          tma_load_2d(smem_u32(sa), ma, fb, kb * BK, m0);
        }
        tma_load_2d(smem_u32(sa + A_BYTES), mb, fb, kb * BK, n0);
      }
    }
    // the last round of each stage has landed before the CTA winds down
    for (uint32_t i = g > (uint32_t)STAGES ? g - STAGES : 0; i < g; ++i)
      mbar_drain(smem_u32(&full[i % STAGES]), (i / STAGES) & 1u);
  } else if (!kHalo && warp == 1 && lane == 0) {
    // ---------------------------------------------------------- MMA issuer
    uint32_t g = 0, q = 0;  // k blocks consumed, chunks produced
    bool alive = true;
    for (int64_t i = 0, t;
         alive && tile_at(order, ostart, blockIdx.x, gridDim.x, total_tiles, i, &t); ++i) {
      const LtbTcProblem& p = probs ? probs[find_problem(probs, nprob, t)] : single;
      const int nk = (int)((p.Kp + BK - 1) / BK);
      for (int c0 = 0, cl = 0; c0 < nk && alive; c0 += cl, ++q) {
        cl = chunk_len(p, c0, nk);
        const int buf = q & 1;
        if (!mbar_wait(smem_u32(&chunk_empty[buf]), ((q >> 1) & 1u) ^ 1u, err)) {
          alive = false;
          break;
        }
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const uint32_t acc = tmem + (uint32_t)(buf * BN);
        const int c1 = c0 + cl;
        for (int kb = c0; kb < c1; ++kb, ++g) {
          const int s = g % STAGES;
          if (!mbar_wait(smem_u32(&full[s]), (g / STAGES) & 1u, err)) {
            alive = false;
            break;
          }
          asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
          const uint32_t a0 = smem_u32(smem + s * STAGE_BYTES);
          const uint64_t ad = sw128_desc(a0), bd = sw128_desc(a0 + A_BYTES);
#pragma unroll
          for (int kk = 0; kk < BK / 16; ++kk)  // +32 bytes per K=16 step
            mma_bf16(acc, ad + 2 * kk, bd + 2 * kk, T::IDESC, (kb != c0) || (kk != 0));
          mma_commit(smem_u32(&empty[s]));  // stage reusable once these finish
        }
        mma_commit(smem_u32(&chunk_full[buf]));  // chunk complete in TMEM
      }
    }
  } else if (warp >= 2) {
    // ------------------------------------------------------ drain/epilogue
    const int quad = warp & 3;            // TMEM lanes 32*quad .. +31
    const int half = (warp - 2) >> 2;     // columns HALF*half .. +HALF-1
    uint32_t q = 0;
    bool alive = true;
    for (int64_t i = 0, t;
         alive && tile_at(order, ostart, blockIdx.x, gridDim.x, total_tiles, i, &t); ++i) {
      const LtbTcProblem& p = probs ? probs[find_problem(probs, nprob, t)] : single;
      int m0, n0;
      tile_coords<BN>(p, t - p.tile_start, &m0, &n0);
      const int nk = (int)((p.Kp + BK - 1) / BK);
      // this thread's output row (row m0 + 32*quad + lane of the tile): its
      // offset is loaded now, its latency hidden behind the chunk waits
      int row;
      const bool rvalid = tile_row(p, m0, quad * 32 + lane, &row);
      const int64_t rbase = rvalid ? p.crow[row] : 0;
      float run[T::HALF];
#pragma unroll
      for (int i = 0; i < T::HALF; ++i) run[i] = 0.f;
      for (int c0 = 0, cl = 0; c0 < nk; c0 += cl, ++q) {
        cl = chunk_len(p, c0, nk);
        const int buf = q & 1;
        const bool ok = mbar_wait(smem_u32(&chunk_full[buf]), (q >> 1) & 1u, err);
        if (!__all_sync(0xffffffffu, ok)) {
          alive = false;
          break;
        }
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const uint32_t base =
            tmem + ((uint32_t)(quad * 32) << 16) + (uint32_t)(buf * BN + half * T::HALF);
        // LD columns per wait: two loads in flight for 128-wide tiles; 256-wide
        // tiles wait after each (their 128 running sums fill the register
        // budget)
        constexpr int LD = BN == 128 ? 32 : 16;
#pragma unroll
        for (int c = 0; c < T::HALF / LD; ++c) {
          uint32_t r[LD];
#pragma unroll
          for (int u = 0; u < LD / 16; ++u) tmem_ld16(base + (uint32_t)(c * LD + u * 16), r + u * 16);
          tmem_wait_ld();
#pragma unroll
          for (int i = 0; i < LD; ++i) run[c * LD + i] += __uint_as_float(r[i]);
        }
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        mbar_arrive(smem_u32(&chunk_empty[buf]));  // buffer free for the MMA
      }
      if (!alive) break;
      // epilogue: this warp owns rows m0 + 32*quad .. +31 (row m0 + 32*quad
      // + lane in this thread's registers) and HALF columns from n0 + half*HALF
      write_tile<T::HALF, kTmaEpi, kTransposeEpi>(
          p, probs ? static_cast<const CUtensorMap*>(p.map_c) : &single_c, c_override, run,
          p.c_tma && !kTransposeEpi ? tma_stage : epi, warp - 2, m0, n0 + half * T::HALF, rvalid,
          rbase);
    }
    if (kTmaEpi && lane == 0) bulk_wait();  // the tile stores have landed
  }
  __syncwarp();
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                 "r"(T::TMEM_COLS));
}

// ------------------------------------------------------------ CTA pairs
// 256 x 256 output tiles on a cluster of two CTAs (tcgen05 cta_group::2):
// CTA rank r loads A rows m0 + 128 r and B' rows n0 + 128 r of every k block
// (16 + 16 KB a stage, its own shared memory), the leader (rank 0) issues
// M = 256, N = 256 MMAs that read both CTAs' stages, and each CTA's TMEM
// receives its own 128 rows of the tile (all 256 columns).  Per SM a k
// block moves 32 KB for the MMA work that costs the single-CTA 128 x 256
// tile 48 KB: the operand stream from L2, not the tensor core, bounds the
// single-CTA form on long K.
//   warp 0 lane 0 (both CTAs): TMA producer; both CTAs' loads complete on
//     the leader's full[s], which alone expects the stage's 64 KB
//   warp 1 lane 0 (leader): MMA issuer; each commit arrives on the barrier
//     at the same offset in both CTAs (empty[s], chunk_full[b])
//   warps 2..9 (both CTAs): drain + epilogue of the CTA's 128 rows; their
//     chunk_empty arrivals go to the leader's barrier (2 x 256 a phase)
// Waits are bounded as in the single-CTA kernel; a cluster barrier after
// set-up and before teardown keeps either CTA from signalling or reading
// the other's shared memory outside its lifetime.
constexpr int kPairStages = 6;
constexpr int kPairStageBytes = 2 * 128 * BK * 2;  // A half + B' half
constexpr size_t kPairSmem = (size_t)kPairStages * kPairStageBytes + 1024 + 256;
constexpr uint32_t kPairTmemCols = 512;  // two 256-column accumulator buffers
// kind::f16: FP32 accumulator, BF16 A and B, both K-major, M = 256, N = 256
constexpr uint32_t kPairIdesc =
    (1u << 4) | (1u << 7) | (1u << 10) | ((256u >> 3) << 17) | ((256u >> 4) << 24);

__device__ __forceinline__ uint32_t cluster_rank() {
  uint32_t r;
  asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
  return r;
}
__device__ __forceinline__ uint32_t cluster_index() {
  uint32_t r;
  asm volatile("mov.u32 %0, %%clusterid.x;" : "=r"(r));
  return r;
}
__device__ __forceinline__ uint32_t cluster_count() {
  uint32_t r;
  asm volatile("mov.u32 %0, %%nclusterid.x;" : "=r"(r));
  return r;
}
// the same shared-memory offset in the cluster's rank-0 CTA
__device__ __forceinline__ uint32_t rank0_addr(uint32_t addr) {
  uint32_t r;
  asm volatile("mapa.shared::cluster.u32 %0, %1, 0;" : "=r"(r) : "r"(addr));
  return r;
}
// every thread of both CTAs
__device__ __forceinline__ void cluster_sync_all() {
  asm volatile("barrier.cluster.arrive.release.aligned;" ::: "memory");
  asm volatile("barrier.cluster.wait.acquire.aligned;" ::: "memory");
}
__device__ __forceinline__ bool mbar_try_cl(uint32_t bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n"
      " mbarrier.try_wait.parity.acquire.cluster.shared::cta.b64 p, [%1], %2;\n"
      " selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
  return ok != 0;
}
// bounded wait on a barrier that other CTAs of the cluster arrive on
__device__ __forceinline__ bool mbar_wait_cl(uint32_t bar, uint32_t parity, int* err) {
  if (mbar_try_cl(bar, parity)) return true;
  const long long t0 = clock64();
  while (!mbar_try_cl(bar, parity)) {
    const long long dt = clock64() - t0;
    if (dt > kWaitCycles || (dt > kFlagCycles && *(volatile int*)err)) {
      atomicExch(err, 1);
      return false;
    }
  }
  return true;
}
__device__ __forceinline__ void mbar_arrive_remote(uint32_t cluster_addr) {
  asm volatile("mbarrier.arrive.release.cluster.shared::cluster.b64 _, [%0];" ::"r"(cluster_addr)
               : "memory");
}
// 2-D TMA load into this CTA's shared memory completing on a barrier of
// either CTA of the pair (cluster address)
__device__ __forceinline__ void tma_load_2d_pair(uint32_t dst, const CUtensorMap* map,
                                                 uint32_t bar, int x, int y) {
  asm volatile(
      "cp.async.bulk.tensor.2d.cta_group::2.shared::cluster.global.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3}], [%4];" ::"r"(dst),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(bar)
      : "memory");
}
__device__ __forceinline__ void mma_bf16_pair(uint32_t tmem_d, uint64_t a, uint64_t b,
                                              uint32_t accumulate) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
      " tcgen05.mma.cta_group::2.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem_d),
      "l"(a), "l"(b), "r"(kPairIdesc), "r"(accumulate));
}
// arrives on the barrier at this offset in both CTAs once the leader's
// MMAs issued so far are complete
__device__ __forceinline__ void mma_commit_pair(uint32_t bar) {
  asm volatile(
      "tcgen05.commit.cta_group::2.mbarrier::arrive::one.shared::cluster.multicast::cluster.b64"
      " [%0], %1;" ::"r"(bar),
      "h"((unsigned short)3)
      : "memory");
}

// Pair tile index -> (m0, n0) of the 256 x 256 tile (tiles_m, tiles_n in
// pair tiles), raster as tile_coords
__device__ __forceinline__ void pair_coords(const LtbTcProblem& p, int64_t lt, int* m0, int* n0) {
  const int gmax = p.group_m > 0 ? p.group_m : 16;
  const int64_t per_group = (int64_t)gmax * p.tiles_n;
  const int g = (int)(lt / per_group);
  const int idx = (int)(lt - (int64_t)g * per_group);
  const int gm = p.tiles_m - g * gmax < gmax ? p.tiles_m - g * gmax : gmax;
  *m0 = (g * gmax + idx % gm) * 256;
  *n0 = (idx / gm) * 256;
}

__global__ void __launch_bounds__(NT, 1)
    k_gemm_tc_pair(const LtbTcProblem* __restrict__ probs, int nprob, int64_t total_tiles,
                   int* err, const int* __restrict__ order, const int* __restrict__ ostart,
                   const __grid_constant__ LtbTcProblem single,
                   const __grid_constant__ CUtensorMap single_a,
                   const __grid_constant__ CUtensorMap single_b,
                   const __grid_constant__ CUtensorMap single_c) {
  extern __shared__ __align__(1024) uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>(
      (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + (size_t)kPairStages * kPairStageBytes);
  uint64_t* empty = full + kPairStages;
  uint64_t* chunk_full = empty + kPairStages;  // [2] MMA -> drain (both CTAs)
  uint64_t* chunk_empty = chunk_full + 2;      // [2] drain -> MMA (the leader's)
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(chunk_empty + 2);
  __shared__ __align__(1024) float epi[8 * 1024];  // drain warps' TMA-store staging
  static_assert(kPairSmem + sizeof(float) * 8 * 1024 <= 227 * 1024, "shared memory per CTA");

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t rank = cluster_rank();
  const bool leader = rank == 0;
  if (threadIdx.x == 0) {
    for (int s = 0; s < kPairStages; ++s) {
      mbar_init(smem_u32(&full[s]), 1);   // the leader's expect_tx
      mbar_init(smem_u32(&empty[s]), 1);  // one commit
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(smem_u32(&chunk_full[b]), 1);
      mbar_init(smem_u32(&chunk_empty[b]), 2 * 8 * 32);  // both CTAs' drain threads
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {  // the same warp in both CTAs allocates for the pair
    asm volatile("tcgen05.alloc.cta_group::2.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(tmem_slot)),
                 "r"(kPairTmemCols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::2.sync.aligned;");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  cluster_sync_all();  // both CTAs' barriers initialised and TMEM allocated
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tmem_slot;
  const int64_t first = cluster_index(), step = cluster_count();

  if (warp == 0 && lane == 0) {
    // ------------------------------------------------------------ producer
    uint32_t g = 0;
    bool alive = true;
    for (int64_t i = 0, t; alive && tile_at(order, ostart, first, step, total_tiles, i, &t);
         ++i) {
      const LtbTcProblem& p = probs ? probs[find_problem(probs, nprob, t)] : single;
      const CUtensorMap* ma = probs ? static_cast<const CUtensorMap*>(p.map_a) : &single_a;
      const CUtensorMap* mb = probs ? static_cast<const CUtensorMap*>(p.map_b) : &single_b;
      int m0, n0;
      pair_coords(p, t - p.tile_start, &m0, &n0);
      const int nk = (int)((p.Kp + BK - 1) / BK);
      for (int kb = 0; kb < nk; ++kb, ++g) {
        const int s = g % kPairStages;
        if (!mbar_wait_cl(smem_u32(&empty[s]), ((g / kPairStages) & 1u) ^ 1u, err)) {
          alive = false;
          break;
        }
        const uint32_t fb = smem_u32(&full[s]);
        if (leader) mbar_expect_tx(fb, 2 * kPairStageBytes);
        const uint32_t sa = smem_u32(smem + (size_t)s * kPairStageBytes);
        const uint32_t fb0 = rank0_addr(fb);
        tma_load_2d_pair(sa, ma, fb0, kb * BK, m0 + 128 * (int)rank);
        tma_load_2d_pair(sa + A_BYTES, mb, fb0, kb * BK, n0 + 128 * (int)rank);
      }
    }
    // the last round of each stage has landed (both CTAs' loads complete on
    // the leader's barriers; the closing cluster barrier holds the peer)
    if (leader)
      for (uint32_t i = g > (uint32_t)kPairStages ? g - kPairStages : 0; i < g; ++i)
        mbar_drain(smem_u32(&full[i % kPairStages]), (i / kPairStages) & 1u);
  } else if (warp == 1 && lane == 0 && leader) {
    // ---------------------------------------------------------- MMA issuer
    uint32_t g = 0, q = 0;
    bool alive = true;
    for (int64_t i = 0, t; alive && tile_at(order, ostart, first, step, total_tiles, i, &t);
         ++i) {
      const LtbTcProblem& p = probs ? probs[find_problem(probs, nprob, t)] : single;
      const int nk = (int)((p.Kp + BK - 1) / BK);
      for (int c0 = 0, cl = 0; c0 < nk && alive; c0 += cl, ++q) {
        cl = chunk_len(p, c0, nk);
        const int buf = q & 1;
        if (!mbar_wait_cl(smem_u32(&chunk_empty[buf]), ((q >> 1) & 1u) ^ 1u, err)) {
          alive = false;
          break;
        }
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const uint32_t acc = tmem + (uint32_t)(buf * 256);
        const int c1 = c0 + cl;
        for (int kb = c0; kb < c1; ++kb, ++g) {
          const int s = g % kPairStages;
          if (!mbar_wait_cl(smem_u32(&full[s]), (g / kPairStages) & 1u, err)) {
            alive = false;
            break;
          }
          asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
          const uint32_t a0 = smem_u32(smem + (size_t)s * kPairStageBytes);
          const uint64_t ad = sw128_desc(a0), bd = sw128_desc(a0 + A_BYTES);
#pragma unroll
          for (int kk = 0; kk < BK / 16; ++kk)
            mma_bf16_pair(acc, ad + 2 * kk, bd + 2 * kk, (kb != c0) || (kk != 0));
          mma_commit_pair(smem_u32(&empty[s]));  // both CTAs' stage s reusable
        }
        mma_commit_pair(smem_u32(&chunk_full[buf]));  // chunk complete in both TMEMs
      }
    }
  } else if (warp >= 2) {
    // ------------------------------------------------------ drain/epilogue
    const int quad = warp & 3, half = (warp - 2) >> 2;
    uint32_t q = 0;
    bool alive = true;
    for (int64_t i = 0, t; alive && tile_at(order, ostart, first, step, total_tiles, i, &t);
         ++i) {
      const LtbTcProblem& p = probs ? probs[find_problem(probs, nprob, t)] : single;
      int m0, n0;
      pair_coords(p, t - p.tile_start, &m0, &n0);
      const int m0c = m0 + 128 * (int)rank;  // this CTA's rows of the tile
      const int nk = (int)((p.Kp + BK - 1) / BK);
      int row;
      const bool rvalid = tile_row(p, m0c, quad * 32 + lane, &row);
      const int64_t rbase = rvalid ? p.crow[row] : 0;
      float run[128];
#pragma unroll
      for (int i = 0; i < 128; ++i) run[i] = 0.f;
      for (int c0 = 0, cl = 0; c0 < nk; c0 += cl, ++q) {
        cl = chunk_len(p, c0, nk);
        const int buf = q & 1;
        const bool ok = mbar_wait_cl(smem_u32(&chunk_full[buf]), (q >> 1) & 1u, err);
        if (!__all_sync(0xffffffffu, ok)) {
          alive = false;
          break;
        }
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const uint32_t base =
            tmem + ((uint32_t)(quad * 32) << 16) + (uint32_t)(buf * 256 + half * 128);
#pragma unroll
        for (int c = 0; c < 8; ++c) {
          uint32_t r[16];
          tmem_ld16(base + (uint32_t)(c * 16), r);
          tmem_wait_ld();
#pragma unroll
          for (int i = 0; i < 16; ++i) run[c * 16 + i] += __uint_as_float(r[i]);
        }
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        mbar_arrive_remote(rank0_addr(smem_u32(&chunk_empty[buf])));  // buffer free
      }
      if (!alive) break;
      write_tile<128, true, false>(p, probs ? static_cast<const CUtensorMap*>(p.map_c) : &single_c,
                                   nullptr, run, epi, warp - 2, m0c, n0 + half * 128, rvalid,
                                   rbase);
    }
    if (lane == 0) bulk_wait();  // the tile stores have landed
  }
  __syncwarp();
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  cluster_sync_all();  // no MMA, commit or arrival of either CTA still in flight
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::2.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                 "r"(kPairTmemCols));
}

// ------------------------------------------------- halo tiles on CTA pairs
// The halo image tiles (weights resident, one 4-D box per tile and channel
// block, every (kh, kw) shift read in place) on a cluster of two CTAs:
// tcgen05.mma.cta_group::2 with M = 256 (the two CTAs' 128-row tiles) and N
// = 128.  CTA rank r holds the box of m-tile 2 pt + r and rows 64 r .. 64 r
// + 63 of every weight block (half of the resident B', 8 KB a block), so
// each SM moves 6 KB of operands per 128 x 128 x 16 product instead of 8
// KB, and loads half of the weights.
//   warp 0 lane 0 (both CTAs): producer; its box and weight loads complete
//     on the leader's barriers, which alone expect both CTAs' bytes
//   warp 1 lane 0 (leader): MMA issuer; commits arrive on the barrier at
//     the same offset in both CTAs (empty[s], chunk_full[b])
//   warps 2..9 (both CTAs): drain + epilogue of the CTA's 128 rows; their
//     chunk_empty arrivals go to the leader's barrier (2 x 256 a phase)
// An odd last m-tile pairs with a tile past the end: its box reads zeros
// (coordinates past the image) and its rows are not written.
constexpr int kPairHaloBBytes = 64 * BK * 2;  // this CTA's half of a weight block
constexpr uint32_t kPairHaloTmemCols = 256;   // two 128-column accumulators
// kind::f16: FP32 accumulator, BF16 A and B, both K-major, M = 256, N = 128
constexpr uint32_t kPairHaloIdesc =
    (1u << 4) | (1u << 7) | (1u << 10) | ((128u >> 3) << 17) | ((256u >> 4) << 24);

__device__ __forceinline__ void tma_load_4d_pair(uint32_t dst, const CUtensorMap* map,
                                                 uint32_t bar, int x, int y, int z, int w) {
  asm volatile(
      "cp.async.bulk.tensor.4d.cta_group::2.shared::cluster.global.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3, %4, %5}], [%6];" ::"r"(dst),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(w), "r"(bar)
      : "memory");
}
__device__ __forceinline__ void mma_bf16_pair_n128(uint32_t tmem_d, uint64_t a, uint64_t b,
                                                   uint32_t accumulate) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
      " tcgen05.mma.cta_group::2.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem_d),
      "l"(a), "l"(b), "r"(kPairHaloIdesc), "r"(accumulate));
}

// Shared memory of a pair-halo CTA: its weight halves, the box ring and the
// barriers (full/empty per slot, one per weight block, 2 + 2 chunk
// barriers, the TMEM address word).
__host__ __device__ inline size_t pair_halo_fixed_bytes(int kbt) {
  return (size_t)kbt * kPairHaloBBytes + 1024 + (size_t)(2 * kMaxHaloStages + kbt + 4) * 8 + 8;
}

__global__ void __launch_bounds__(NT, 1)
    k_gemm_tc_pair_halo(int64_t pair_tiles, int* err, const __grid_constant__ LtbTcProblem single,
                        const __grid_constant__ CUtensorMap single_a,
                        const __grid_constant__ CUtensorMap single_b) {
  const LtbTcProblem& p = single;
  extern __shared__ __align__(1024) uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>(
      (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  const int kbt = (int)(p.Kp / BK), nst = p.img_stages;
  const uint32_t slot_bytes = (uint32_t)p.img_slot_bytes;
  uint8_t* bres = smem;  // weight block kb's half at bres + kb * 8 KB
  uint8_t* ring = smem + (size_t)kbt * kPairHaloBBytes;
  uint64_t* full = reinterpret_cast<uint64_t*>(ring + (size_t)nst * slot_bytes);
  uint64_t* empty = full + nst;
  uint64_t* b_full = empty + nst;            // [kbt] (the leader's count both halves)
  uint64_t* chunk_full = b_full + kbt;       // [2] MMA -> drain (both CTAs)
  uint64_t* chunk_empty = chunk_full + 2;    // [2] drain -> MMA (the leader's)
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(chunk_empty + 2);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t rank = cluster_rank();
  const bool leader = rank == 0;
  if (threadIdx.x == 0) {
    for (int s = 0; s < nst; ++s) {
      mbar_init(smem_u32(&full[s]), 1);   // the leader's expect_tx
      mbar_init(smem_u32(&empty[s]), 1);  // one commit
    }
    for (int kb = 0; kb < kbt; ++kb) mbar_init(smem_u32(&b_full[kb]), 1);
    for (int b = 0; b < 2; ++b) {
      mbar_init(smem_u32(&chunk_full[b]), 1);
      mbar_init(smem_u32(&chunk_empty[b]), 2 * 8 * 32);  // both CTAs' drain threads
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {  // the same warp in both CTAs allocates for the pair
    asm volatile("tcgen05.alloc.cta_group::2.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(tmem_slot)),
                 "r"(kPairHaloTmemCols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::2.sync.aligned;");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  cluster_sync_all();  // both CTAs' barriers initialised and TMEM allocated
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tmem_slot;
  const int64_t first = cluster_index(), step = cluster_count();
  const int ncb = p.img_cblocks, nsh = p.img_kh * p.img_kw;

  if (warp == 0 && lane == 0) {
    // ------------------------------------------------------------ producer
    const uint32_t box_bytes = (uint32_t)((p.img_rows + p.img_kh - 1) * p.img_slot * 128);
    bool first_tile = true;  // the first tile also loads the weight halves, in first-use order
    uint32_t g = 0;          // stages issued
    bool alive = true;
    for (int64_t pt = first; pt < pair_tiles && alive; pt += step) {
      const int mt = (int)(2 * pt) + (int)rank;  // halo tiles: one column of tiles, no raster
      const int n_img = mt / p.img_hgroups;
      const int ho0 = (mt - n_img * p.img_hgroups) * p.img_rows;
      for (int cb = 0; cb < ncb; ++cb, ++g) {
        const int s = (int)(g % (uint32_t)nst);
        if (!mbar_wait_cl(smem_u32(&empty[s]), ((g / (uint32_t)nst) & 1u) ^ 1u, err)) {
          alive = false;
          break;
        }
        if (first_tile)
          for (int sh = 0; sh < nsh; ++sh) {
            const int kb = sh * ncb + cb;
            const uint32_t bb = smem_u32(&b_full[kb]);
            if (leader) mbar_expect_tx(bb, 2u * kPairHaloBBytes);
            tma_load_2d_pair(smem_u32(bres + (size_t)kb * kPairHaloBBytes), &single_b,
                             rank0_addr(bb), kb * BK, 64 * (int)rank);
          }
        const uint32_t fb = smem_u32(&full[s]);
        if (leader) mbar_expect_tx(fb, 2u * box_bytes);
        tma_load_4d_pair(smem_u32(ring + (size_t)s * slot_bytes), &single_a, rank0_addr(fb),
                         cb * 64, 0, ho0, n_img);
      }
      first_tile = false;
    }
    // both CTAs' loads complete on the leader's barriers: the leader waits
    // for the last round of each slot and the weight blocks loaded (those
    // of the first tile's first g channel blocks); the closing cluster
    // barrier holds the peer until then
    if (leader) {
      for (uint32_t i = g > (uint32_t)nst ? g - nst : 0; i < g; ++i)
        mbar_drain(smem_u32(&full[i % nst]), (i / nst) & 1u);
      for (int kb = 0; kb < kbt; ++kb)
        if ((uint32_t)(kb % ncb) < g) mbar_drain(smem_u32(&b_full[kb]), 0u);
    }
  } else if (warp == 1 && lane == 0 && leader) {
    // ---------------------------------------------------------- MMA issuer
    uint32_t g = 0, q = 0;  // stages consumed, chunks produced
    bool alive = true;
    bool first_tile = true;  // weight blocks are waited for on first use
    constexpr int cbk = kChunkBlocks;
    const uint64_t a_kh = (uint64_t)p.img_slot * 8u;  // descriptor steps, 16-byte units
    const uint64_t b_blk = (uint64_t)(kPairHaloBBytes >> 4), b_shift = (uint64_t)ncb * b_blk;
    const uint64_t b0 = sw128_desc(smem_u32(bres));
    for (int64_t pt = first; pt < pair_tiles && alive; pt += step) {
      int issued = 0, buf = 0;
      uint32_t acc = tmem;
      for (int cb = 0; cb < ncb && alive; ++cb, ++g) {
        const int s = (int)(g % (uint32_t)nst);
        if (!mbar_wait_cl(smem_u32(&full[s]), (g / (uint32_t)nst) & 1u, err)) {
          alive = false;
          break;
        }
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        uint64_t arow = sw128_desc(smem_u32(ring + (size_t)s * slot_bytes));
        uint64_t bd = b0 + (uint64_t)cb * b_blk;
        int kb = cb;
        for (int kh = 0; kh < p.img_kh && alive; ++kh, arow += a_kh)
          for (int kw = 0; kw < p.img_kw; ++kw, bd += b_shift, kb += ncb) {
            if (issued % cbk == 0) {  // a new accumulation chunk
              buf = (int)(q & 1u);
              if (!mbar_wait_cl(smem_u32(&chunk_empty[buf]), ((q >> 1) & 1u) ^ 1u, err)) {
                alive = false;
                break;
              }
              asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
              acc = tmem + (uint32_t)(buf * 128);
            }
            if (first_tile && !mbar_wait_cl(smem_u32(&b_full[kb]), 0u, err)) {
              alive = false;
              break;
            }
            const uint64_t ad = arow + 8u * (uint64_t)kw;
#pragma unroll
            for (int kk = 0; kk < BK / 16; ++kk)
              mma_bf16_pair_n128(acc, ad + 2 * kk, bd + 2 * kk, (issued % cbk != 0) || (kk != 0));
            ++issued;
            if (issued % cbk == 0 || issued == kbt) {
              mma_commit_pair(smem_u32(&chunk_full[buf]));  // chunk complete in both TMEMs
              ++q;
            }
          }
        mma_commit_pair(smem_u32(&empty[s]));  // both CTAs' slot s reusable
      }
      first_tile = false;
    }
  } else if (warp >= 2) {
    // ------------------------------------------------------ drain/epilogue
    const int quad = warp & 3, half = (warp - 2) >> 2;
    uint32_t q = 0;
    bool alive = true;
    for (int64_t pt = first; pt < pair_tiles && alive; pt += step) {
      const int mt = (int)(2 * pt) + (int)rank;
      const int m0 = mt * BM;
      int row;
      const bool rvalid = mt < p.tiles_m && tile_row(p, m0, quad * 32 + lane, &row);
      const int64_t rbase = rvalid ? p.crow[row] : 0;
      float run[64];
#pragma unroll
      for (int i = 0; i < 64; ++i) run[i] = 0.f;
      for (int c0 = 0; c0 < kbt; c0 += kChunkBlocks, ++q) {
        const int buf = q & 1;
        const bool ok = mbar_wait_cl(smem_u32(&chunk_full[buf]), (q >> 1) & 1u, err);
        if (!__all_sync(0xffffffffu, ok)) {
          alive = false;
          break;
        }
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const uint32_t base =
            tmem + ((uint32_t)(quad * 32) << 16) + (uint32_t)(buf * 128 + half * 64);
#pragma unroll
        for (int c = 0; c < 2; ++c) {
          uint32_t r[32];
          tmem_ld16(base + (uint32_t)(c * 32), r);
          tmem_ld16(base + (uint32_t)(c * 32 + 16), r + 16);
          tmem_wait_ld();
#pragma unroll
          for (int i = 0; i < 32; ++i) run[c * 32 + i] += __uint_as_float(r[i]);
        }
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        mbar_arrive_remote(rank0_addr(smem_u32(&chunk_empty[buf])));  // buffer free
      }
      if (!alive) break;
      write_tile<64, false, false>(p, nullptr, nullptr, run, nullptr, warp - 2, m0, half * 64,
                                   rvalid, rbase);
    }
  }
  __syncwarp();
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  cluster_sync_all();  // no MMA, commit or arrival of either CTA still in flight
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::2.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                 "r"(kPairHaloTmemCols));
}

// ------------------------------------------------------------ packing
// Gathers an operand through its separable description and writes the BF16
// split of every element into nseg K-segments of a K-major matrix: bit s of
// seg_mask selects the hi part (1) or the lo part (0, x - hi rounded to
// BF16) for segment s, bit 8 + s the third part (x - hi - lo).  Columns
// [nseg*K, Kp) of every row are zeroed (the packed buffers live in reused
// scratch).
//
// Work unit: a 64-row x 64-k tile.  Each CTA takes a contiguous range of
// tiles (one job search per CTA, sequential addresses).  Four load modes:
//   kPackDenseK   dense, k-contiguous: float4 loads, 16-byte BF16 stores,
//                 no shared memory
//   kPackDenseR   dense, row-contiguous (B[k, n] feeding B'[n, k]): float4
//                 loads along rows into a swizzled shared tile (no bank
//                 conflicts), transposed on the way out
//   kPackGatherK / kPackGatherR  guarded gathers (padding, views), lanes
//                 along k or along rows, through the shared tile
constexpr int PR = 64, PKT = 64, PACK_THREADS = 256;

// 8 consecutive k of row r (k < K) split and stored into every segment.
// The pieces of x: hi = bf16(x), lo = bf16(x - hi), lo2 = bf16(x - hi - lo);
// each difference is exact in FP32, and lo2 holds the last bits, so
// hi + lo + lo2 == x for normal x.  Segment s takes lo2 when bit 8 + s of
// seg_mask is set, else hi (bit s set) or lo.
__device__ __forceinline__ void pack_store8(const LtbPackJob& J, int64_t r, int64_t k,
                                            const float (&x)[8]) {
  uint32_t hi[4], lo[4], lo2[4];
  const bool third = (J.seg_mask >> 8) != 0;
#pragma unroll
  for (int e = 0; e < 4; ++e) {
    const __nv_bfloat162 h = __floats2bfloat162_rn(x[2 * e], x[2 * e + 1]);
    const float2 hf = __bfloat1622float2(h);
    const float r0 = x[2 * e] - hf.x, r1 = x[2 * e + 1] - hf.y;
    const __nv_bfloat162 l = __floats2bfloat162_rn(r0, r1);
    hi[e] = *reinterpret_cast<const uint32_t*>(&h);
    lo[e] = *reinterpret_cast<const uint32_t*>(&l);
    if (third) {
      const float2 lf = __bfloat1622float2(l);
      const __nv_bfloat162 l2 = __floats2bfloat162_rn(r0 - lf.x, r1 - lf.y);
      lo2[e] = *reinterpret_cast<const uint32_t*>(&l2);
    } else {
      lo2[e] = 0;
    }
  }
  __nv_bfloat16* out = static_cast<__nv_bfloat16*>(J.out);
  const int nv = J.K - k < 8 ? (int)(J.K - k) : 8;
  const uint4 H = make_uint4(hi[0], hi[1], hi[2], hi[3]);
  const uint4 L = make_uint4(lo[0], lo[1], lo[2], lo[3]);
  const uint4 L2 = make_uint4(lo2[0], lo2[1], lo2[2], lo2[3]);
  for (int s = 0; s < J.nseg; ++s) {
    const uint4 v = (J.seg_mask >> (8 + s)) & 1 ? L2 : (J.seg_mask >> s) & 1 ? H : L;
    const int64_t off = r * J.Kp + s * J.K + k;
    if (nv == 8 && (off & 7) == 0) {
      *reinterpret_cast<uint4*>(out + off) = v;
    } else {
      const uint32_t w[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
      for (int e = 0; e < 8; ++e)
        if (e < nv) {
          const unsigned short b = (unsigned short)(w[e >> 1] >> (16 * (e & 1)));
          out[off + e] = __ushort_as_bfloat16(b);
        }
    }
  }
}

static_assert(sizeof(LtbPackJob) % 8 == 0, "job copied as 8-byte words");

struct PackTables {
  int64_t roff[PR], koff[PKT];
  int32_t roff32[PR], koff32[PKT];  // the same offsets when the job is off32
  int32_t grow[LTB_MAXG][PR], gk[LTB_MAXG][PKT], gub[LTB_MAXG];
};

// Guarded gather of one 64 x 64 tile into sm[k][r].  One side of the
// element grid is fixed per thread (64 divides the block), so its offset
// and guard partials stay in registers; the other side is warp-uniform and
// read from the staged tables (broadcast).  NG: guard count (-1: any, up to
// LTB_MAXG, through a runtime loop).
template <int NG, bool along_r, bool off32>
__device__ __forceinline__ void gather_fill(const LtbPackJob& J, const PackTables& tb,
                                            float (*sm)[PR + 1], int64_t rlim, int64_t klim,
                                            int ng) {
  constexpr int G = NG < 0 ? LTB_MAXG : NG;
  const int tid = threadIdx.x;
  const int fixed = tid & 63;
  const bool fok = fixed < (along_r ? rlim : klim);
  const int64_t fo = off32 ? (int64_t)(along_r ? tb.roff32[fixed] : tb.koff32[fixed])
                           : (along_r ? tb.roff[fixed] : tb.koff[fixed]);
  const int32_t fo32 = (int32_t)fo;
  const int vlim = (int)(along_r ? klim : rlim);
  int32_t fg[G > 0 ? G : 1], ub[G > 0 ? G : 1];
#pragma unroll
  for (int g = 0; g < G; ++g) {
    const bool on = NG >= 0 || g < ng;
    fg[g] = on ? (along_r ? tb.grow[g][fixed] : tb.gk[g][fixed]) : 0;
    ub[g] = on ? tb.gub[g] : 1;  // off: 0 <= 0 + 0 < 1 always holds
  }
  // all 16 gathers issue before any shared-memory store (loads in flight)
  float v[16];
#pragma unroll
  for (int q = 0; q < 16; ++q) {
    const int v_ = (tid >> 6) + 4 * q;  // the varying side (warp-uniform)
    v[q] = 0.f;
    if (fok && v_ < vlim) {
      bool ok = true;
#pragma unroll
      for (int g = 0; g < G; ++g) {  // 0 <= w < ub as one unsigned compare
        const int32_t o = NG >= 0 || g < ng ? (along_r ? tb.gk[g][v_] : tb.grow[g][v_]) : 0;
        ok = ok && (uint32_t)(fg[g] + o) < (uint32_t)ub[g];
      }
      if (ok) {
        if (off32)
          v[q] = __ldg(J.op.base +
                       (uint32_t)(fo32 + (along_r ? tb.koff32[v_] : tb.roff32[v_])));
        else
          v[q] = __ldg(J.op.base + fo + (along_r ? tb.koff[v_] : tb.roff[v_]));
      }
    }
  }
#pragma unroll
  for (int q = 0; q < 16; ++q) {
    const int v_ = (tid >> 6) + 4 * q;
    if (along_r) sm[v_][fixed] = v[q];
    else sm[fixed][v_] = v[q];
  }
}

// kDense: the dense modes alone (a launch whose every job is dense); the
// gather branch is compiled out, so the kernel fits more CTAs per SM.
template <bool kDense>
__device__ __forceinline__ void pack_tile(const LtbPackJob& J, int64_t lt,
                                          float (*sm)[PR + 1], PackTables* tabs) {
  const int tid = threadIdx.x;
  int64_t rt, kt;  // tile row / k indices (32-bit division when it fits)
  if (lt <= 0xffffffffLL) {
    const uint32_t q = (uint32_t)lt / (uint32_t)J.tiles_k;
    rt = q;
    kt = (uint32_t)lt - q * (uint32_t)J.tiles_k;
  } else {
    rt = lt / J.tiles_k;
    kt = lt - rt * J.tiles_k;
  }
  const int64_t r0 = rt * PR, k0 = kt * PKT;
  if (J.mode == kPackDenseK) {
    float x[2][8];
#pragma unroll
    for (int i = 0; i < 2; ++i) {
      const int64_t r = r0 + (tid >> 3) + 32 * i, k = k0 + (tid & 7) * 8;
      const bool rok = r < J.rows;
      const float* p = J.op.base + r * J.op.ld_row + k;
      const float4 z = make_float4(0.f, 0.f, 0.f, 0.f);
      const float4 u = rok && k < J.K ? __ldg(reinterpret_cast<const float4*>(p)) : z;
      const float4 v = rok && k + 4 < J.K ? __ldg(reinterpret_cast<const float4*>(p + 4)) : z;
      x[i][0] = u.x; x[i][1] = u.y; x[i][2] = u.z; x[i][3] = u.w;
      x[i][4] = v.x; x[i][5] = v.y; x[i][6] = v.z; x[i][7] = v.w;
    }
#pragma unroll
    for (int i = 0; i < 2; ++i) {
      const int64_t r = r0 + (tid >> 3) + 32 * i, k = k0 + (tid & 7) * 8;
      if (r < J.rows && k < J.K) pack_store8(J, r, k, x[i]);
    }
  } else if (J.mode == kPackDenseR) {
    // Transposed through the shared tile viewed as [64 k][64 r] floats with
    // r stored at r ^ 4 * ((k / 8) % 8): the float4 writes of a quarter-warp
    // (one k, 32 consecutive r) fill one 128-byte line, and the 8 reads of
    // a thread (8 consecutive k of one r, k / 8 differing across the warp)
    // hit 32 distinct banks -- no bank conflicts either way.  Loads: a warp
    // reads two k rows of 64 contiguous floats; stores: 8 threads write one
    // row's 64 k (128 bytes of BF16).
    float* t = &sm[0][0];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int idx = tid + PACK_THREADS * q;
      const int kl = idx >> 4, rl = (idx & 15) * 4;
      const int64_t k = k0 + kl, r = r0 + rl;
      float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
      if (k < J.K && r < J.rows)  // rows % 4 == 0 in this mode
        v = __ldg(reinterpret_cast<const float4*>(J.op.base + k * J.op.ld_k + r));
      *reinterpret_cast<float4*>(t + kl * 64 + (rl ^ ((kl >> 3) << 2))) = v;
    }
    __syncthreads();
#pragma unroll
    for (int i = 0; i < 2; ++i) {
      const int c = tid + PACK_THREADS * i;
      const int rl = c >> 3, kc = c & 7;
      const int64_t r = r0 + rl, k = k0 + kc * 8;
      if (r < J.rows && k < J.K) {
        float x[8];
#pragma unroll
        for (int e = 0; e < 8; ++e) x[e] = t[(kc * 8 + e) * 64 + (rl ^ (kc << 2))];
        pack_store8(J, r, k, x);
      }
    }
    __syncthreads();  // the next tile overwrites the shared tile
  } else {
    // shared tile sm[k][r], row pitch 65 floats
    if constexpr (!kDense) {
      // guarded gather: the tile's row and k tables staged in shared memory
      // (offsets and guard partials), so each element costs one global load
      PackTables& tb = *tabs;
      const int ng = J.op.dense ? 0 : J.op.nguard;
      if (tid < 64) {
        const int64_t k = k0 + tid;
        const bool ok = k < J.K;
        tb.koff[tid] = !ok ? 0 : J.op.dense ? k * J.op.ld_k : J.op.koff[k];
        tb.koff32[tid] = (int32_t)tb.koff[tid];
        for (int g = 0; g < ng; ++g) tb.gk[g][tid] = ok ? J.op.gk[(int64_t)g * J.K + k] : 0;
      } else if (tid < 128) {
        const int rl = tid - 64;
        const int64_t r = r0 + rl;
        const bool ok = r < J.rows;
        tb.roff[rl] = !ok ? 0 : J.op.dense ? r * J.op.ld_row : J.op.rowoff[r];
        tb.roff32[rl] = (int32_t)tb.roff[rl];
        for (int g = 0; g < ng; ++g) tb.grow[g][rl] = ok ? J.op.grow[(int64_t)g * J.rows + r] : 0;
      } else if (tid < 128 + LTB_MAXG) {
        if (tid - 128 < ng) tb.gub[tid - 128] = J.op.gub[tid - 128];
      }
      __syncthreads();
      const int64_t rlim = J.rows - r0, klim = J.K - k0;
      const bool along_r = J.mode == kPackGatherR;
#define LTB_GATHER(AR, O32)                                                    \
  switch (ng) { /* guard count known at compile time: no predicated loop */      \
    case 0: gather_fill<0, AR, O32>(J, tb, sm, rlim, klim, ng); break;          \
    case 1: gather_fill<1, AR, O32>(J, tb, sm, rlim, klim, ng); break;          \
    case 2: gather_fill<2, AR, O32>(J, tb, sm, rlim, klim, ng); break;          \
    case 3: gather_fill<3, AR, O32>(J, tb, sm, rlim, klim, ng); break;          \
    case 4: gather_fill<4, AR, O32>(J, tb, sm, rlim, klim, ng); break;          \
    default: gather_fill<-1, AR, O32>(J, tb, sm, rlim, klim, ng); break;        \
  }
      if (along_r) {
        if (J.off32) {
          LTB_GATHER(true, true)
        } else {
          LTB_GATHER(true, false)
        }
      } else {
        if (J.off32) {
          LTB_GATHER(false, true)
        } else {
          LTB_GATHER(false, false)
        }
      }
#undef LTB_GATHER
    }
    __syncthreads();
#pragma unroll
    for (int i = 0; i < 2; ++i) {
      const int c = tid + PACK_THREADS * i;
      const int rl = c >> 3, kc = c & 7;
      const int64_t r = r0 + rl, k = k0 + kc * 8;
      if (r < J.rows && k < J.K) {
        float x[8];
#pragma unroll
        for (int e = 0; e < 8; ++e) x[e] = sm[kc * 8 + e][rl];
        pack_store8(J, r, k, x);
      }
    }
    __syncthreads();  // the next tile overwrites sm
  }
  if (k0 == 0) {  // K padding [nseg*K, Kp) of this tile's rows
    const int pad = (int)(J.Kp - J.nseg * J.K);
    __nv_bfloat16* out = static_cast<__nv_bfloat16*>(J.out);
    for (int c = tid; c < PR * pad; c += PACK_THREADS) {
      const int64_t r = r0 + c / pad;
      if (r < J.rows) out[r * J.Kp + J.nseg * J.K + c % pad] = __float2bfloat16_rn(0.f);
    }
  }
}

__device__ __forceinline__ void tile_range(int64_t total, int64_t& t0, int64_t& t1) {
  t0 = total * blockIdx.x / gridDim.x;
  t1 = total * (blockIdx.x + 1) / gridDim.x;
}

// Dense launches can hold 6 CTAs per SM (40 registers, no spills), half as
// many loads again in flight as the general form's 4; single-segment (BF16)
// packing runs them (8192^2 operands: 156 -> 137 us), the split modes, whose
// stores outnumber their loads, keep 4 (measured slower with 6).
constexpr int kPackCtasDense = 6, kPackCtas = 4;

template <bool kDense>
__global__ void __launch_bounds__(PACK_THREADS, kDense ? kPackCtasDense : kPackCtas)
    k_pack_one(const __grid_constant__ LtbPackJob J, int64_t total_tiles) {
  __shared__ float sm[PKT][PR + 1];
  PackTables* tabs = nullptr;  // the gather tables (general form only)
  if constexpr (!kDense) {
    __shared__ PackTables tb;
    tabs = &tb;
  }
  int64_t t0, t1;
  tile_range(total_tiles, t0, t1);
  for (int64_t t = t0; t < t1; ++t) pack_tile<kDense>(J, t, sm, tabs);
}

// Every operand of a batch in one launch; the job of a tile is found by
// binary search on tile_start once per CTA, then by stepping forward.
template <bool kDense>
__global__ void __launch_bounds__(PACK_THREADS, kDense ? kPackCtasDense : kPackCtas)
    k_pack_grouped(const LtbPackJob* __restrict__ jobs, int njobs, int64_t total_tiles,
                   int kGroupChunk) {
  __shared__ float sm[PKT][PR + 1];
  PackTables* tabs = nullptr;  // the gather tables (general form only)
  if constexpr (!kDense) {
    __shared__ PackTables tb;
    tabs = &tb;
  }
  __shared__ LtbPackJob sj;  // the current job, read from shared memory
  // chunks of kGroupChunk consecutive tiles dealt round-robin to the CTAs:
  // every CTA sees a mix of the jobs (fast and slow layouts alike), and its
  // tile indices only grow, so the job index only moves forward
  const int64_t nchunks = (total_tiles + kGroupChunk - 1) / kGroupChunk;
  int64_t ch = blockIdx.x;
  if (ch >= nchunks) return;
  int j = 0, hi = njobs - 1, cur = -1;
  const int64_t t_first = ch * kGroupChunk;
  while (j < hi) {
    const int mid = (j + hi + 1) >> 1;
    if (jobs[mid].tile_start <= t_first) j = mid;
    else hi = mid - 1;
  }
  // first tile of the next job, kept in a register: the job table is read
  // only when a job ends (streaming operand loads would evict it from L1)
  int64_t next_start = j + 1 < njobs ? __ldg(&jobs[j + 1].tile_start) : total_tiles;
  for (; ch < nchunks; ch += gridDim.x) {
    const int64_t t1 = (ch + 1) * kGroupChunk < total_tiles ? (ch + 1) * kGroupChunk
                                                             : total_tiles;
    for (int64_t t = ch * kGroupChunk; t < t1; ++t) {
      if (t >= next_start) {  // skip ahead (binary search)
        int lo = j + 1, h2 = njobs - 1;
        while (lo < h2) {
          const int mid = (lo + h2 + 1) >> 1;
          if (__ldg(&jobs[mid].tile_start) <= t) lo = mid;
          else h2 = mid - 1;
        }
        j = lo;
        next_start = j + 1 < njobs ? __ldg(&jobs[j + 1].tile_start) : total_tiles;
      }
      if (j != cur) {  // uniform across the block
        __syncthreads();
        const uint64_t* src = reinterpret_cast<const uint64_t*>(jobs + j);
        for (int i = threadIdx.x; i < (int)(sizeof(LtbPackJob) / 8); i += PACK_THREADS)
          reinterpret_cast<uint64_t*>(&sj)[i] = src[i];
        __syncthreads();
        cur = j;
      }
      // a register copy of the job: fields read through shared memory on
      // every use cost the tile loop a quarter of its speed
      const LtbPackJob Jl = sj;
      pack_tile<kDense>(Jl, t - Jl.tile_start, sm, tabs);
    }
  }
}

// Image operand repack: one CTA per (channel block of 64, padded row, image)
// reads the 64 channel rows of x (coalesced along w) into shared memory and
// writes the padded row [wp, 64] of BF16 channel pairs (coalesced along c)
// into the hi image, and into the lo and lo2 images when the job has them.
// The reads of a chunk of CJ 32-column slices are all issued before any is
// stored (8 x CJ loads in flight per thread); CJ = ceil(wp / 32) up to 5,
// so a narrow image keeps no idle slices and few registers, and more of its
// rows are in flight on an SM.
template <int CJ>
__device__ __forceinline__ void pack_image_row(const LtbImageJob& J, int cb, int h, int n,
                                               float* tile /* [64][wp + 1] */) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int pitch = J.wp + 1;
  const int hs = h + J.off_h;  // source row
  const bool row_ok = hs >= 0 && hs < J.ub_h;
  // warp per channel row (8 rows per warp), lanes along the columns
  const float* src = J.base + J.off + (int64_t)n * J.ns + (int64_t)(cb * 64 + warp) * J.cs +
                     (int64_t)h * J.wx;
  for (int w0 = 0; w0 < J.wp; w0 += 32 * CJ) {
    float v[8][CJ];
#pragma unroll
    for (int i = 0; i < 8; ++i)
#pragma unroll
      for (int j = 0; j < CJ; ++j) {
        const int w = w0 + lane + 32 * j, ws = w + J.off_w;
        v[i][j] = row_ok && w < J.wp && ws >= 0 && ws < J.ub_w
                      ? __ldg(src + (int64_t)(8 * i) * J.cs + w)
                      : 0.f;
      }
#pragma unroll
    for (int i = 0; i < 8; ++i)
#pragma unroll
      for (int j = 0; j < CJ; ++j) {
        const int w = w0 + lane + 32 * j;
        if (w < J.wp) tile[(warp + 8 * i) * pitch + w] = v[i][j];
      }
  }
  __syncthreads();
  // warp per padded column, lanes over channel pairs (coalesced 128-byte rows)
  __nv_bfloat16* hi = static_cast<__nv_bfloat16*>(J.hi) +
                      (((int64_t)n * J.hp + h) * J.wp) * J.c + cb * 64 + 2 * lane;
  const int64_t at = (((int64_t)n * J.hp + h) * J.wp) * J.c + cb * 64 + 2 * lane;
  __nv_bfloat16* lo = J.lo ? static_cast<__nv_bfloat16*>(J.lo) + at : nullptr;
  __nv_bfloat16* lo2 = J.lo && J.lo2 ? static_cast<__nv_bfloat16*>(J.lo2) + at : nullptr;
  for (int w = warp; w < J.wp; w += 8) {
    const float x0 = tile[2 * lane * pitch + w], x1 = tile[(2 * lane + 1) * pitch + w];
    const __nv_bfloat162 hv = __floats2bfloat162_rn(x0, x1);
    *reinterpret_cast<__nv_bfloat162*>(hi + (int64_t)w * J.c) = hv;
    if (lo) {
      // the pieces of pack_store8: both differences are exact in FP32
      const float2 hf = __bfloat1622float2(hv);
      const float r0 = x0 - hf.x, r1 = x1 - hf.y;
      const __nv_bfloat162 lv = __floats2bfloat162_rn(r0, r1);
      *reinterpret_cast<__nv_bfloat162*>(lo + (int64_t)w * J.c) = lv;
      if (lo2) {
        const float2 lf = __bfloat1622float2(lv);
        *reinterpret_cast<__nv_bfloat162*>(lo2 + (int64_t)w * J.c) =
            __floats2bfloat162_rn(r0 - lf.x, r1 - lf.y);
      }
    }
  }
}

template <int CJ>
__global__ void __launch_bounds__(256) k_pack_image(const __grid_constant__ LtbImageJob J) {
  extern __shared__ float tile[];  // [64][wp + 1]
  pack_image_row<CJ>(J, blockIdx.x, blockIdx.y, blockIdx.z, tile);
}

// 32-column slices per repack chunk for a padded width
inline int image_chunk_slices(int wp) { return wp <= 32 ? 1 : wp <= 64 ? 2 : wp <= 128 ? 4 : 5; }

// A convolution's two operands in one launch: the first nb CTAs pack the
// weight tiles (B'), the rest repack one image row each; the small weight
// job runs beside the image instead of as a launch of its own.
template <int CJ>
__global__ void __launch_bounds__(256, CJ <= 2 ? 5 : 3)
    k_pack_conv(const __grid_constant__ LtbImageJob J, const __grid_constant__ LtbPackJob JB,
                int64_t b_tiles, int nb) {
  extern __shared__ float tile[];  // image: [64][wp + 1]; weights: [64][65]
  __shared__ PackTables tabs;
  const int b = blockIdx.x;
  if (b < nb) {
    const int64_t t0 = b_tiles * b / nb, t1 = b_tiles * (b + 1) / nb;
    for (int64_t t = t0; t < t1; ++t)
      pack_tile<false>(JB, t, reinterpret_cast<float (*)[PR + 1]>(tile), &tabs);
    return;
  }
  const int cblocks = J.c / 64, r = (b - nb) / cblocks;
  pack_image_row<CJ>(J, (b - nb) - r * cblocks, r % J.hp, r / J.hp, tile);
}

PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  if (!fn) {
    cudaDriverEntryPointQueryResult q;
    void* p = nullptr;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  }
  return fn;
}

}  // namespace

cudaError_t ltb_make_tmap(void* map, const void* base, int64_t rows, int64_t Kp, int box_rows) {
  auto fn = encode_fn();
  if (!fn) return cudaErrorNotSupported;
  const cuuint64_t dims[2] = {(cuuint64_t)Kp, (cuuint64_t)rows};
  const cuuint64_t strides[1] = {(cuuint64_t)Kp * 2};
  const cuuint32_t box[2] = {(cuuint32_t)BK, (cuuint32_t)box_rows};
  const cuuint32_t estr[2] = {1, 1};
  CUresult r = fn(reinterpret_cast<CUtensorMap*>(map), CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2,
                  const_cast<void*>(base), dims, strides, box, estr,
                  CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                  CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS ? cudaSuccess : cudaErrorInvalidValue;
}

cudaError_t ltb_make_tmap_c(void* map, float* base, int64_t M, int64_t N, int64_t ld) {
  auto fn = encode_fn();
  if (!fn || M < 1 || N < 1 || ld < N || ld % 4 || reinterpret_cast<uintptr_t>(base) % 16)
    return cudaErrorInvalidValue;
  const cuuint64_t dims[2] = {(cuuint64_t)N, (cuuint64_t)M};
  const cuuint64_t strides[1] = {(cuuint64_t)ld * 4};
  const cuuint32_t box[2] = {32, 32};
  const cuuint32_t estr[2] = {1, 1};
  CUresult r = fn(reinterpret_cast<CUtensorMap*>(map), CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, base,
                  dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                  CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_NONE,
                  CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS ? cudaSuccess : cudaErrorInvalidValue;
}

cudaError_t ltb_make_tmap_image(void* map, const void* base, int n, int hp, int wp, int c,
                                int wo, int rows) {
  auto fn = encode_fn();
  if (!fn || c % 64 || wo < 1 || wo > 256 || rows < 1 || rows > 256) return cudaErrorInvalidValue;
  const cuuint64_t dims[4] = {(cuuint64_t)c, (cuuint64_t)wp, (cuuint64_t)hp, (cuuint64_t)n};
  const cuuint64_t strides[3] = {(cuuint64_t)c * 2, (cuuint64_t)wp * c * 2,
                                 (cuuint64_t)hp * wp * c * 2};
  const cuuint32_t box[4] = {64, (cuuint32_t)wo, (cuuint32_t)rows, 1};
  const cuuint32_t estr[4] = {1, 1, 1, 1};
  CUresult r = fn(reinterpret_cast<CUtensorMap*>(map), CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 4,
                  const_cast<void*>(base), dims, strides, box, estr,
                  CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                  CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS ? cudaSuccess : cudaErrorInvalidValue;
}

bool ltb_tc_halo_geometry(LtbTcProblem& p, int wp) {
  if (!p.img || p.N > 128 || p.Kp % BK || wp > 128 || p.Kp / BK > kMaxHaloKb) return false;
  // the (kh, kw)-shifted operand reads box rows kh * wp + kw .. + 127
  const int slot_bytes = (((p.img_kh - 1) * wp + 127 + p.img_kw) * 128 + 1023) / 1024 * 1024;
  const size_t fixed = (size_t)(p.Kp / BK) * kHaloBBytes + 1024 + kHaloBarBytes;
  if (fixed + 2 * (size_t)slot_bytes > kHaloSmemMax) return false;
  int stages = (int)((kHaloSmemMax - fixed) / slot_bytes);
  stages = stages < kMaxHaloStages ? stages : kMaxHaloStages;
  const int nimg = p.tiles_m / p.img_hgroups;  // per-row form: tiles_m = nimg * hgroups
  p.img_halo = 1;
  p.img_slot = wp;
  p.img_rows = 128 / wp;
  p.img_hgroups = (p.img_ho + p.img_rows - 1) / p.img_rows;
  p.tiles_m = nimg * p.img_hgroups;
  p.tiles_n = 1;
  p.img_stages = stages;
  p.img_slot_bytes = slot_bytes;
  return true;
}

cudaError_t ltb_launch_pack_image(const LtbImageJob& j, cudaStream_t st) {
  if (j.c % 64 || j.wp < 1 || j.wp > 1024) return cudaErrorInvalidValue;
  const size_t smem = (size_t)64 * (j.wp + 1) * sizeof(float);
  const dim3 grid((unsigned)(j.c / 64), (unsigned)j.hp, (unsigned)j.nimg);
#define LTB_IMG(CJ)                                                                       \
  {                                                                                       \
    if (smem > 48 * 1024) {                                                               \
      const cudaError_t e = ltb_smem_optin((const void*)k_pack_image<CJ>, smem);          \
      if (e != cudaSuccess) return e;                                                     \
    }                                                                                     \
    k_pack_image<CJ><<<grid, 256, smem, st>>>(j);                                         \
    return cudaGetLastError();                                                            \
  }
  switch (image_chunk_slices(j.wp)) {
    case 1: LTB_IMG(1)
    case 2: LTB_IMG(2)
    case 4: LTB_IMG(4)
    default: LTB_IMG(5)
  }
#undef LTB_IMG
}

static LtbPackJob make_pack_job(const LtbGemmOperand& op, int64_t rows, int64_t K, void* out,
                                int64_t Kp, int nseg, int seg_mask, int k_contig, int off32);

cudaError_t ltb_launch_pack_conv(const LtbImageJob& j, const LtbGemmOperand& bop, int64_t rows,
                                 int64_t K, void* out, int64_t Kp, int nseg, int seg_mask,
                                 int k_contig, int off32, cudaStream_t st) {
  if (j.c % 64 || j.wp < 1 || j.wp > 1024) return cudaErrorInvalidValue;
  const LtbPackJob JB = make_pack_job(bop, rows, K, out, Kp, nseg, seg_mask, k_contig, off32);
  const int64_t b_tiles = ltb_pack_tiles(rows, K);
  const int64_t img_ctas = (int64_t)(j.c / 64) * j.hp * j.nimg;
  const int nb = (int)(b_tiles < 64 ? b_tiles : 64);
  if (img_ctas + nb > 0x7fffffff) return cudaErrorInvalidValue;
  size_t smem = (size_t)64 * (j.wp + 1) * sizeof(float);
  if (smem < (size_t)PKT * (PR + 1) * sizeof(float)) smem = (size_t)PKT * (PR + 1) * sizeof(float);
#define LTB_CONV(CJ)                                                                      \
  {                                                                                       \
    if (smem > 40 * 1024) { /* 48 KB less the static pack tables */                       \
      const cudaError_t e = ltb_smem_optin((const void*)k_pack_conv<CJ>, smem);           \
      if (e != cudaSuccess) return e;                                                     \
    }                                                                                     \
    k_pack_conv<CJ><<<(unsigned)(img_ctas + nb), 256, smem, st>>>(j, JB, b_tiles, nb);    \
    return cudaGetLastError();                                                            \
  }
  switch (image_chunk_slices(j.wp)) {
    case 1: LTB_CONV(1)
    case 2: LTB_CONV(2)
    case 4: LTB_CONV(4)
    default: LTB_CONV(5)
  }
#undef LTB_CONV
}

int ltb_tc_tile_m() { return BM; }

int ltb_pack_mode(const LtbGemmOperand& op, int64_t rows, int64_t K, int k_contig) {
  const bool aligned = (reinterpret_cast<uintptr_t>(op.base) & 15) == 0;
  if (op.dense && aligned && op.ld_k == 1 && (op.ld_row & 3) == 0 && (K & 3) == 0)
    return kPackDenseK;
  if (op.dense && aligned && op.ld_row == 1 && (op.ld_k & 3) == 0 && (rows & 3) == 0)
    return kPackDenseR;
  return k_contig ? kPackGatherK : kPackGatherR;
}

int64_t ltb_pack_tiles(int64_t rows, int64_t K) {
  return ((rows + PR - 1) / PR) * ((K + PKT - 1) / PKT);
}

static int64_t pack_grid(int64_t tiles, int sms, bool dense_one_segment) {
  const int64_t g = (int64_t)sms * (dense_one_segment ? kPackCtasDense : kPackCtas);
  return tiles < g ? tiles : g;
}

static bool pack_dense(int mode) { return mode == kPackDenseK || mode == kPackDenseR; }

static LtbPackJob make_pack_job(const LtbGemmOperand& op, int64_t rows, int64_t K, void* out,
                                int64_t Kp, int nseg, int seg_mask, int k_contig, int off32) {
  LtbPackJob J{};
  J.op = op;
  J.out = out;
  J.rows = rows;
  J.K = K;
  J.Kp = Kp;
  J.tiles_k = (int)((K + PKT - 1) / PKT);
  J.nseg = nseg;
  J.seg_mask = seg_mask;
  J.mode = ltb_pack_mode(op, rows, K, k_contig);
  J.off32 = off32;
  return J;
}

cudaError_t ltb_launch_pack(const LtbGemmOperand& op, int64_t rows, int64_t K, void* out,
                            int64_t Kp, int nseg, int seg_mask, int k_contig, int off32, int sms,
                            cudaStream_t st) {
  const LtbPackJob J = make_pack_job(op, rows, K, out, Kp, nseg, seg_mask, k_contig, off32);
  const int64_t tiles = ltb_pack_tiles(rows, K);
  if (tiles == 0) return cudaSuccess;
  if (pack_dense(J.mode))
    k_pack_one<true><<<(unsigned)pack_grid(tiles, sms, nseg == 1), PACK_THREADS, 0, st>>>(J,
                                                                                       tiles);
  else
    k_pack_one<false><<<(unsigned)pack_grid(tiles, sms, false), PACK_THREADS, 0, st>>>(J, tiles);
  return cudaGetLastError();
}

cudaError_t ltb_launch_pack_grouped(const LtbPackJob* d_jobs, int njobs, int64_t total_tiles,
                                    int sms, cudaStream_t st, int chunk, int cta_per_sm,
                                    int all_dense, int all_one_segment) {
  if (total_tiles == 0) return cudaSuccess;
  if (chunk < 1) chunk = 4;
  const int64_t chunks = (total_tiles + chunk - 1) / chunk;
  const int per_sm = cta_per_sm > 0                        ? cta_per_sm
                     : all_dense && all_one_segment ? kPackCtasDense
                                                            : kPackCtas;
  const int64_t cap = (int64_t)sms * per_sm;
  const int64_t grid = chunks < cap ? chunks : cap;
  if (all_dense)
    k_pack_grouped<true><<<(unsigned)grid, PACK_THREADS, 0, st>>>(d_jobs, njobs, total_tiles,
                                                                  chunk);
  else
    k_pack_grouped<false><<<(unsigned)grid, PACK_THREADS, 0, st>>>(d_jobs, njobs, total_tiles,
                                                                   chunk);
  return cudaGetLastError();
}

static size_t halo_smem(const LtbTcProblem& p) {
  return (size_t)(p.Kp / BK) * kHaloBBytes + (size_t)p.img_stages * p.img_slot_bytes + 1024 +
         kHaloBarBytes;
}

template <int BN, bool TE, int CTAS = 1, bool HALO = false>
static cudaError_t launch_tc(const LtbTcProblem* d_probs, int nprob, int64_t total_tiles,
                             float* c_override, int sms, int* err, cudaStream_t st,
                             const LtbTcProblem* single, const void* map_a, const void* map_b,
                             const void* map_a2, const void* map_a3, const void* map_c,
                             bool c_tma_any, const int* order = nullptr,
                             const int* ostart = nullptr) {
  // TMA-stored outputs in this launch: the staging in dynamic shared memory
  const bool tma = !TE && CTAS == 1 && !HALO && (d_probs ? c_tma_any : single && single->c_tma && map_c);
  size_t smem = tma ? Tile<BN, CTAS>::SMEM_TMA : Tile<BN, CTAS>::SMEM;
  if (HALO) {
    if (d_probs || !single || !single->img_halo) return cudaErrorInvalidValue;
    smem = halo_smem(*single);
    if (smem > kHaloSmemMax) return cudaErrorInvalidValue;
  }
  {
    const cudaError_t e = ltb_smem_optin(
        (const void*)k_gemm_tc<BN, TE, CTAS, HALO>,
        HALO ? kHaloSmemMax : !TE && CTAS == 1 ? Tile<BN, CTAS>::SMEM_TMA : smem);
    if (e != cudaSuccess) return e;
  }
  const int64_t slots = (int64_t)sms * CTAS;
  const int grid = (int)(total_tiles < slots ? total_tiles : slots);
  LtbTcProblem one{};
  CUtensorMap ma{}, mb{}, ma2{}, ma3{}, mc{};
  if (!d_probs) {
    if (!single || !map_a || !map_b) return cudaErrorInvalidValue;
    one = *single;
    ma = *static_cast<const CUtensorMap*>(map_a);
    mb = *static_cast<const CUtensorMap*>(map_b);
    ma2 = map_a2 ? *static_cast<const CUtensorMap*>(map_a2) : ma;
    ma3 = map_a3 ? *static_cast<const CUtensorMap*>(map_a3) : ma2;
    if (map_c) mc = *static_cast<const CUtensorMap*>(map_c);
    else one.c_tma = 0;
  }
  k_gemm_tc<BN, TE, CTAS, HALO><<<grid, NT, smem, st>>>(d_probs, nprob, total_tiles, c_override,
                                                        err, order, ostart, one, ma, mb, ma2, ma3,
                                                        mc);
  return cudaGetLastError();
}

// Clusters of two CTAs a pair kernel can hold resident at once on a device
// with this much dynamic shared memory (its persistent grid): asked once per
// kernel, size and device.
static int pair_clusters(const void* fn, size_t smem, int dev) {
  static std::mutex mu;
  static std::map<std::tuple<const void*, size_t, int>, int> known;
  std::lock_guard<std::mutex> g(mu);
  const auto key = std::make_tuple(fn, smem, dev);
  auto it = known.find(key);
  if (it != known.end()) return it->second;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(2, 1, 1);
  cfg.blockDim = dim3(NT, 1, 1);
  cfg.dynamicSmemBytes = smem;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeClusterDimension;
  at[0].val.clusterDim.x = 2;
  at[0].val.clusterDim.y = 1;
  at[0].val.clusterDim.z = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  int n = 0;
  if (cudaOccupancyMaxActiveClusters(&n, fn, &cfg) != cudaSuccess) {
    cudaGetLastError();
    n = 0;
  }
  known[key] = n;
  return n;
}

static cudaError_t launch_pair(const LtbTcProblem* d_probs, int nprob, int64_t total_tiles,
                               int* err, cudaStream_t st, const LtbTcProblem* single,
                               const void* map_a, const void* map_b, const void* map_c,
                               const int* order, const int* ostart) {
  {
    const cudaError_t e = ltb_smem_optin((const void*)k_gemm_tc_pair, kPairSmem);
    if (e != cudaSuccess) return e;
  }
  int dev = 0;
  {
    const cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
  }
  int64_t clusters = pair_clusters((const void*)k_gemm_tc_pair, kPairSmem, dev);
  if (clusters <= 0) return cudaErrorInvalidConfiguration;
  if (total_tiles < clusters) clusters = total_tiles;
  LtbTcProblem one{};
  CUtensorMap ma{}, mb{}, mc{};
  if (!d_probs) {
    if (!single || !map_a || !map_b || single->img) return cudaErrorInvalidValue;
    one = *single;
    ma = *static_cast<const CUtensorMap*>(map_a);
    mb = *static_cast<const CUtensorMap*>(map_b);
    if (map_c) mc = *static_cast<const CUtensorMap*>(map_c);
    else one.c_tma = 0;
  }
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)(2 * clusters), 1, 1);
  cfg.blockDim = dim3(NT, 1, 1);
  cfg.dynamicSmemBytes = kPairSmem;
  cfg.stream = st;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeClusterDimension;
  at[0].val.clusterDim.x = 2;
  at[0].val.clusterDim.y = 1;
  at[0].val.clusterDim.z = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, k_gemm_tc_pair, d_probs, nprob, total_tiles, err, order, ostart,
                            one, ma, mb, mc);
}

// Halo tiles on CTA pairs: the halo problem with the ring re-sized for the
// halved weight residency; tiles = its m-tiles, run two to a cluster.
static cudaError_t launch_pair_halo(int64_t tiles, int* err, cudaStream_t st,
                                    const LtbTcProblem* single, const void* map_a,
                                    const void* map_b) {
  if (!single || !single->img_halo || !map_a || !map_b || single->N > 128)
    return cudaErrorInvalidValue;
  LtbTcProblem one = *single;
  const int kbt = (int)(one.Kp / BK);
  const size_t fixed = pair_halo_fixed_bytes(kbt);
  if (kbt > kMaxHaloKb || fixed + 2 * (size_t)one.img_slot_bytes > kHaloSmemMax)
    return cudaErrorInvalidValue;
  const int stages = (int)((kHaloSmemMax - fixed) / (size_t)one.img_slot_bytes);
  one.img_stages = stages < kMaxHaloStages ? stages : kMaxHaloStages;
  const size_t smem = fixed + (size_t)one.img_stages * (size_t)one.img_slot_bytes;
  {
    const cudaError_t e = ltb_smem_optin((const void*)k_gemm_tc_pair_halo, kHaloSmemMax);
    if (e != cudaSuccess) return e;
  }
  int dev = 0;
  {
    const cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
  }
  int64_t clusters = pair_clusters((const void*)k_gemm_tc_pair_halo, smem, dev);
  if (clusters <= 0) return cudaErrorInvalidConfiguration;
  const int64_t pair_tiles = (tiles + 1) / 2;
  if (pair_tiles < clusters) clusters = pair_tiles;
  const CUtensorMap ma = *static_cast<const CUtensorMap*>(map_a);
  const CUtensorMap mb = *static_cast<const CUtensorMap*>(map_b);
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)(2 * clusters), 1, 1);
  cfg.blockDim = dim3(NT, 1, 1);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeClusterDimension;
  at[0].val.clusterDim.x = 2;
  at[0].val.clusterDim.y = 1;
  at[0].val.clusterDim.z = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, k_gemm_tc_pair_halo, pair_tiles, err, one, ma, mb);
}

int64_t ltb_tc_units(int bn, int64_t total_tiles, int sms) {
  if (total_tiles <= 0) return 0;
  int64_t units = (int64_t)sms * (bn == 130 ? 2 : 1);
  if (bn == 258) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) {
      cudaGetLastError();
      return 0;
    }
    units = pair_clusters((const void*)k_gemm_tc_pair, kPairSmem, dev);
  }
  return total_tiles < units ? total_tiles : units;
}

cudaError_t ltb_launch_gemm_tc(int bn, const LtbTcProblem* d_probs, int nprob,
                               int64_t total_tiles, float* c_override, int sms, int* err,
                               cudaStream_t st, const LtbTcProblem* single, const void* map_a,
                               const void* map_b, const void* map_a2, const void* map_a3,
                               const void* map_c, int c_tma_any, const int* order,
                               const int* ostart) {
  if (total_tiles == 0) return cudaSuccess;
  if (order && bn != 128 && bn != 129 && bn != 256 && bn != 257 && bn != 130 && bn != 258)
    return cudaErrorInvalidValue;  // an order is for the batch (problem-table) forms
#define LTB_TC(BN, TE)                                                                      \
  return launch_tc<BN, TE>(d_probs, nprob, total_tiles, c_override, sms, err, st, single, map_a, \
                           map_b, map_a2, map_a3, map_c, c_tma_any, order, ostart)
  switch (bn) {
    case 128: LTB_TC(128, false);
    case 129: LTB_TC(128, true);
    case 256: LTB_TC(256, false);
    case 257: LTB_TC(256, true);
    case 130:  // 128 wide, two CTAs per SM
      return launch_tc<128, false, 2>(d_probs, nprob, total_tiles, c_override, sms, err, st,
                                      single, map_a, map_b, map_a2, map_a3, map_c, false, order,
                                      ostart);
    case 131:  // 128 wide halo image tiles, resident weights
      return launch_tc<128, false, 1, true>(d_probs, nprob, total_tiles, c_override, sms, err,
                                            st, single, map_a, map_b, map_a2, map_a3, map_c,
                                            false);
    case 258:  // 256 x 256 tiles on CTA pairs (plain operands, B' boxes of 128 rows)
      if (c_override) return cudaErrorInvalidValue;
      return launch_pair(d_probs, nprob, total_tiles, err, st, single, map_a, map_b, map_c,
                         order, ostart);
    case 133:  // halo image tiles on CTA pairs (M = 256, B' boxes of 64 rows)
      if (c_override || d_probs) return cudaErrorInvalidValue;
      return launch_pair_halo(total_tiles, err, st, single, map_a, map_b);
  }
#undef LTB_TC
  return cudaErrorInvalidValue;
}
