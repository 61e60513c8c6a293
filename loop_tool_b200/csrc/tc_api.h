// Host API of the tcgen05 contraction kernels (gemm_tc.cu).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "kernels.h"

// One GEMM problem of a (possibly grouped) persistent launch.  Lives in
// device memory; map_a / map_b point at CUtensorMaps in device memory.
struct LtbTcProblem {
  const void* map_a;     // CUtensorMap over A' [M, Kp] BF16 K-major
  const void* map_b;     // CUtensorMap over B' [N, Kp] BF16 K-major
  float* c;
  const int64_t* crow;   // [M] output row offsets
  const int64_t* ccol;   // [N] output column offsets (unused if unit_cols)
  int64_t Kp;
  int64_t tile_start;    // first global tile index of this problem
  int M, N;
  int tiles_m, tiles_n;
  int unit_cols;         // ccol[j] == j
  int group_m;           // raster: row blocks swept together (0: 16)
  // Output by TMA stores: C rows are an arithmetic progression
  // (crow[r] = crow[0] + r * ld, ld % 4 == 0) of unit columns, and map_c is
  // a CUtensorMap over C + crow[0] (ltb_make_tmap_c); single-CTA plain tiles
  // only (0: per-thread row stores)
  int c_tma;
  const void* map_c;
  // Image operand (implicit-GEMM convolution, stride 1): A is read straight
  // from a zero-padded NHWC BF16 image [n, Hp, Wp, C] through 4-D boxes of
  // 64 channels x wo output columns, one box per output image row; a
  // 128-row tile holds img_rows image rows of img_slot rows each (wo
  // rounded up to 8), i.e. output rows m = (n * ho + h) * wo + w.  K runs
  // (kh, kw, c): k-block = (kh * kw_n + kw) * cblocks + channel block.
  int img;               // 0: A' [M, Kp] dense as above
  int img_rows, img_slot, img_wo, img_ho, img_hgroups;
  int img_kh, img_kw, img_cblocks;
  int img_a_mask;        // bit s: segment s reads the hi image (1) or lo (0);
                         // bit 8 + s: segment s reads the lo2 image
  const void* map_a2;    // image mode: CUtensorMap over the lo image
  const void* map_a3;    // image mode: CUtensorMap over the lo2 image
  // Halo image tiles (single-segment image operands, N <= 128, single
  // launches): img_slot = the padded width wp, so tile row i * wp + w is
  // output column w of image row i; one 4-D box of img_rows padded rows per
  // (kh, channel block) stage, and the kw shifts of that box are read by the
  // MMA at row offsets of kw * 128 bytes.  B' stays resident in shared
  // memory (every k block loaded once per CTA).
  int img_halo;
  int img_stages;        // halo ring depth
  int img_slot_bytes;    // bytes per halo ring slot (1024-aligned)
  // 64-wide k blocks accumulated into one TMEM buffer before the drain
  // warps add it into FP32 registers (0: 8).  The tensor core's FP32
  // accumulation truncates, so its error grows with the MMA steps of a
  // chunk: the FP32-accurate split modes drain shorter chunks.
  int chunk_blocks;
  // Past the first main_blocks k blocks, chunks of rest_blocks when set
  // (0: chunk_blocks throughout): the six-product mode's correction
  // segments, whose products are 2^-8 of the main segment's and whose
  // truncation is as far below it, drain in longer chunks.
  int main_blocks, rest_blocks;
};

// Repacks an image operand x(n, c, h + off_h, w + off_w) (FP32 at
// base + n*ns + c*cs + h*wx + w, element (h, w) of the window valid iff
// 0 <= h + off_h < ub_h and 0 <= w + off_w < ub_w, else 0) into zero-padded
// NHWC BF16 images [n, hp, wp, c]: the hi part into hi, the lo part
// (x - hi rounded to BF16) into lo when lo is not null.
struct LtbImageJob {
  const float* base;     // the operand's buffer; element (n,c,h,w) at base + off
  int64_t off, ns, cs, wx;
  int nimg, c, hp, wp;
  int off_h, ub_h, off_w, ub_w;
  void* hi;
  void* lo;   // x - hi, rounded (null: hi only)
  void* lo2;  // (x - hi) - lo, rounded (null: no third piece; needs lo)
};
cudaError_t ltb_launch_pack_image(const LtbImageJob& j, cudaStream_t st);
// The image repack and the B' packing of the same contraction (arguments
// as ltb_launch_pack) in one launch.
cudaError_t ltb_launch_pack_conv(const LtbImageJob& j, const LtbGemmOperand& bop, int64_t rows,
                                 int64_t K, void* out, int64_t Kp, int nseg, int seg_mask,
                                 int k_contig, int off32, cudaStream_t st);
// CUtensorMap over an FP32 output [M, N] with row pitch ld (floats) in
// 32 x 32 boxes, 128-byte swizzled: base 16-byte aligned, ld % 4 == 0.
cudaError_t ltb_make_tmap_c(void* map, float* base, int64_t M, int64_t N, int64_t ld);
// CUtensorMap over an NHWC BF16 image [n, hp, wp, c] with boxes of
// 64 channels x wo columns x rows image rows (128-byte swizzle):
// c % 64 == 0, wo <= 256, rows <= 256.
cudaError_t ltb_make_tmap_image(void* map, const void* base, int n, int hp, int wp, int c,
                                int wo, int rows = 1);
// Halo tile geometry of an image problem (fills img_halo, img_slot,
// img_rows, img_hgroups, tiles_m, img_stages, img_slot_bytes of p from its
// per-row form); false if the weights or the ring do not fit in shared
// memory.
bool ltb_tc_halo_geometry(LtbTcProblem& p, int img_wp);

// Load modes of the operand packer (ltb_pack_mode picks one per operand).
enum { kPackDenseK = 0, kPackDenseR = 1, kPackGatherK = 2, kPackGatherR = 3 };

// One operand packing job: FP32 operand -> BF16 K-major [rows, Kp] in
// 64-row x 64-k tiles.
struct LtbPackJob {
  LtbGemmOperand op;
  void* out;            // BF16 [rows, Kp]
  int64_t rows, K, Kp;
  int64_t tile_start;   // first global tile index of this job (grouped launch)
  int tiles_k;          // ceil(K / 64)
  int nseg, seg_mask;
  int mode;             // kPack*
  int off32;            // every element offset of the operand fits in int32
  int pad_;
};
int ltb_pack_mode(const LtbGemmOperand& op, int64_t rows, int64_t K, int k_contig);
int64_t ltb_pack_tiles(int64_t rows, int64_t K);
// Tiles are dealt to the CTAs in round-robin chunks of `chunk` consecutive
// tiles (0: 4); grid = SMs x cta_per_sm CTAs (0: 4, or 6 when every job is
// of a dense mode with one segment).  all_dense selects the kernel without
// the gather path.
cudaError_t ltb_launch_pack_grouped(const LtbPackJob* d_jobs, int njobs, int64_t total_tiles,
                                    int sms, cudaStream_t st, int chunk = 0, int cta_per_sm = 0,
                                    int all_dense = 0, int all_one_segment = 0);

// CUtensorMap (128 bytes, 64-byte aligned) over a K-major BF16 matrix
// [rows, Kp] (Kp a multiple of 8 so the row pitch is 16-byte aligned),
// boxes of 64 x box_rows with 128-byte swizzle.
cudaError_t ltb_make_tmap(void* map, const void* base, int64_t rows, int64_t Kp, int box_rows);

// FP32 operand -> BF16 K-major segments (hi / lo split per segment).
// off32: every element offset (rowoff[r] + koff[k], both >= 0) is below 2^31,
// so the gather adds 32-bit offsets.
cudaError_t ltb_launch_pack(const LtbGemmOperand& op, int64_t rows, int64_t K, void* out,
                            int64_t Kp, int nseg, int seg_mask, int k_contig, int off32, int sms,
                            cudaStream_t st);

// Persistent grouped launch over every tile of every problem
// (tiles_m * ceil(N / tile) tiles per problem, tile = bn & ~1 = 128 or 256:
// the tile width the problems' tiles_n and B tensor maps were made for;
// odd bn selects the epilogue that transposes 32 x 32 blocks through shared
// memory into whole-row stores instead of per-thread 16-byte row stores;
// 130: 128 wide, two CTAs per SM; 131: 128 wide halo image tiles with
// resident weights, single problems only).
// c_override, if not null, replaces every problem's output pointer.
// d_probs == nullptr: a single problem passed by value with its tensor maps
// (host copies, passed as kernel parameters; no map_c: row stores).
// c_tma_any: some problem of d_probs has c_tma set (the launch reserves the
// TMA-store staging).
// order / ostart (device arrays, batch forms only): the tiles of work unit u
// (a CTA, or a cluster of two for 258) are order[ostart[u] .. ostart[u+1]),
// for ltb_tc_units(bn, total_tiles, sms) units; without them unit u takes
// tiles u, u + units, ...
cudaError_t ltb_launch_gemm_tc(int bn, const LtbTcProblem* d_probs, int nprob,
                               int64_t total_tiles, float* c_override, int sms, int* err,
                               cudaStream_t st, const LtbTcProblem* single = nullptr,
                               const void* map_a = nullptr, const void* map_b = nullptr,
                               const void* map_a2 = nullptr, const void* map_a3 = nullptr,
                               const void* map_c = nullptr, int c_tma_any = 0,
                               const int* order = nullptr, const int* ostart = nullptr);
// Work units (CTAs, or CTA pairs for 258) of the persistent launch of a
// batch form over total_tiles tiles on this device.
int64_t ltb_tc_units(int bn, int64_t total_tiles, int sms);
int ltb_tc_tile_m();
