/*
 * loop_tool_b200: C ABI of the B200 (sm_100a) "cuda" backend for loop_tool.
 *
 * The boundary is the reference plugin surface, loop_tool's
 * include/loop_tool/backend.h: a Backend compiles a LoopTree into a
 * Compiled, whose run(memory, sync) executes it over caller-owned buffers.
 * A LoopTree crosses this ABI as the text serialize() writes
 * (src/core/serialization.cpp:175-237): the IR, its per-node loop orders
 * (splits, tails), reuse flags and loop annotations, from which the
 * reference rebuilds the identical LoopTree (include/loop_tool/ir.h:402).
 *
 * Conventions (same as the reference):
 *  - memory[] = [inputs in IR input order..., outputs in IR output order...]
 *    as float* (src/core/compile.cpp:506-525).  Pointers may be device,
 *    managed or plain host memory; host buffers are staged through HBM.
 *  - scratch is owned by the compiled object (src/backends/cpu/cpp.cpp:482).
 *  - errors: the reference throws std::runtime_error through ASSERT
 *    (include/loop_tool/error.h:47-61); here every call returns a status and
 *    ltb_last_error() holds the message for the calling thread.
 */
#ifndef LOOP_TOOL_B200_H_
#define LOOP_TOOL_B200_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define LTB_OK 0
#define LTB_ERR_INVALID 1      /* malformed IR text or bad argument */
#define LTB_ERR_UNSUPPORTED 2  /* IR outside what the backend lowers */
#define LTB_ERR_CUDA 3         /* CUDA runtime / launch failure */
#define LTB_ERR_NO_DEVICE 4    /* no usable sm_100 device */
#define LTB_ERR_TIMEOUT 5      /* a bounded device wait gave up */

typedef struct ltb_compiled ltb_compiled;
typedef struct ltb_batch ltb_batch;

/* ABI version (increments on incompatible change). */
int ltb_abi_version(void);

/* Message of the last failed call on this thread ("" if none). */
const char* ltb_last_error(void);

/* Number of visible sm_100 devices.  The reference registers its "cuda"
 * backend and hardware only when a device is present
 * (src/backends/cuda/cuda.cpp:1030-1041); callers do the same with this. */
int ltb_device_count(void);

/* Lowering only, no device needed: writes the kernel plan chosen for the
 * serialized LoopTree into buf (NUL-terminated, truncated to len).
 * Replaces the host-side analysis of cuda_code_and_dispatch /
 * calc_cuda_aux (src/backends/cuda/cuda.cpp:776-792, 973-1028).
 * options: "precision=fp32|bf16|bf16x3|bf16x4;fuse_rows=0|1;tensor_cores=0|1".
 * fp32: CUDA-core FP32 contractions; bf16: BF16 tensor cores, FP32
 * accumulation; bf16x3 / bf16x4: split-BF16 with 3 / 4 products. */
int ltb_plan(const char* ir_text, const char* options, char* buf, size_t len);

/* Backend::compile(const LoopTree&) (include/loop_tool/backend.h:62-67),
 * i.e. CudaBackend::compile_impl (src/backends/cuda/cuda.cpp:875-879):
 * lowers the serialized LoopTree, uploads kernel descriptors and allocates
 * scratch on the current device. */
int ltb_compile(const char* ir_text, const char* options, ltb_compiled** out);

/* Compiled::run(const std::vector<void*>& memory, bool sync)
 * (include/loop_tool/backend.h:20-21; CudaCompiled::run,
 * src/backends/cuda/cuda.cpp:837-850).  stream: a cudaStream_t or NULL for
 * the legacy default stream.  With sync == 0 the call returns after
 * enqueueing (Compiled::async, backend.h:41-44); host buffers are then
 * written back by stream-ordered copies, complete once the stream is (pin
 * them for the copies to overlap).  Runs whose every buffer is in host
 * memory and whose loop tree is one linear elementwise map stage their
 * copies chunk by chunk on two streams (uploads overlap downloads).
 * Managed buffers are prefetched to the device before the launch and, for
 * sync != 0, the outputs back to the host after it (bulk migration instead
 * of demand paging; the reference frontend reads results on the host).
 * Runs of one compiled object on its own (default) scratch are ordered on
 * the device: a run waits for the previous such run, whatever its stream,
 * before its kernels touch the scratch.  With sync != 0 a bounded wait that
 * gave up in a kernel on this stream is reported as LTB_ERR_TIMEOUT. */
int ltb_run(ltb_compiled* c, void* const* memory, int n, int sync,
            void* stream);

/* Like ltb_run with caller-provided scratch (ltb_int_property
 * "scratch_bytes" bytes, 256-byte aligned device memory), so concurrent runs
 * of one compiled object on different streams do not share scratch. */
int ltb_run_with_scratch(ltb_compiled* c, void* const* memory, int n,
                         int sync, void* stream, void* scratch);

/* How ltb_run would treat each buffer, one line per buffer, decided on the
 * host without launching anything: device memory of the compiled object's
 * device and managed memory are read and written in place when 16-byte
 * aligned (the kernels move 16-byte vectors and the tensor-core packers
 * feed the TMA engine); host memory and device/managed memory off a 16-byte
 * boundary (e.g. a view starting one element into a tensor) are staged
 * through an aligned device copy; another GPU's memory is rejected
 * (LTB_ERR_INVALID) rather than read as a peer.  Captured runs, batches and
 * the autotuner take in-place buffers only.  No reference counterpart: the
 * reference's Compiled::run (backend.h:20-21) passes pointers as given. */
int ltb_run_plan(ltb_compiled* c, void* const* memory, int n, char* buf,
                 size_t len);

/* Compiled destructor. */
int ltb_release(ltb_compiled* c);

/* Compiled::dump() / string_properties["code"]
 * (src/backends/cuda/cuda.cpp:970): the kernel plan, not PTX. */
int ltb_dump(ltb_compiled* c, char* buf, size_t len);

/* Compiled::int_properties (src/backends/cuda/cuda.cpp:960-969):
 * "bandwidth" (theoretical GB/s, 2*memclk*buswidth/8 as the reference
 * computes it), plus "stages", "launches", "scratch_bytes", "inputs",
 * "outputs", "algorithmic_bytes", "flops", "tuned" (schedules from the
 * autotuner or its cache), "implicit_conv" (contractions whose A operand is
 * read as an image: convolution as implicit GEMM), "tma_store_output"
 * (tensor-core contractions whose output rows are one progression of
 * 16-byte multiples, written by TMA stores when the buffer is aligned). */
int ltb_int_property(ltb_compiled* c, const char* name, int64_t* value);

/* Element counts of the I/O buffers: elems[0..n_in+n_out). */
int ltb_io_sizes(ltb_compiled* c, int* n_in, int* n_out, int64_t* elems,
                 int cap);

/* Hardware "cuda" (CudaGPUHardware, src/backends/cuda/cuda.cpp:800-816):
 * managed == 1 is cudaMallocManaged like the reference (CPU compatible);
 * managed == 2 is pinned host memory (also CPU and GPU compatible: runs
 * stage it through HBM with overlapped copies, and the CPU reads and writes
 * it without page migration -- faster when every run's inputs are written
 * and its outputs read on the host); managed == 0 is plain device memory.
 * ltb_free releases any of them. */
int ltb_alloc(size_t bytes, int managed, void** out);
int ltb_free(void* ptr);

/* Batches of contractions.  No single counterpart in the reference, which
 * runs one loop tree per Compiled::run (backend.h:20-21); a batch runs n
 * compiled single-contraction loop trees (e.g. matmuls of uneven sizes,
 * one precision) as one grouped launch -- one operand-packing launch and one
 * persistent tensor-core launch over every tile of every problem (FP32: one
 * grouped CUDA-core launch).  memories[i] are the device buffers of member
 * i in Compiled::run order, bound at creation. */
int ltb_batch_create(ltb_compiled* const* cs, void* const* const* memories, int n,
                     ltb_batch** out);
/* Records the batch's launches once into a CUDA graph (stream must not be
 * the legacy default stream); later ltb_batch_run calls replay it. */
int ltb_batch_capture(ltb_batch* b, void* stream);
int ltb_batch_run(ltb_batch* b, int sync, void* stream);
/* One eager run with device timings of its two phases (operand packing and
 * the grouped GEMM), measured with CUDA events on `stream`; synchronises. */
int ltb_batch_run_timed(ltb_batch* b, void* stream, float* pack_ms, float* gemm_ms);
/* Launch shape of the batch's grouped operand packing: tiles dealt to the
 * CTAs in round-robin chunks of pack_chunk consecutive 64x64 tiles, grid =
 * SMs x pack_cta_per_sm (0: the defaults, 4 and 4).  Drops a captured graph
 * (capture again). */
int ltb_batch_set_schedule(ltb_batch* b, int pack_chunk, int pack_cta_per_sm);
/* "problems", "flops", "launches", "tiles", "tiles_128", "tiles_256",
 * "tiles_pair" (256 x 256 tiles on CTA pairs), "graph", "pack_chunk",
 * "pack_cta_per_sm". */
int ltb_batch_int_property(ltb_batch* b, const char* name, int64_t* value);
int ltb_batch_release(ltb_batch* b);

/* Row sums out[r] = sum_c x[r * cols + c] (row-major x[rows, cols]) that
 * allocate nothing.  No counterpart in the reference: it is for callers that
 * cannot allocate device memory when they call in -- a serving loop that
 * committed its whole HBM budget up front, or a host framework that owns
 * every device allocation -- and it equals ltb_run on the loop tree
 * (X.sum(n)) within FP32 rounding.  x and out must be device or managed
 * memory.  Split-K partials live in one static device array of 2^20 floats
 * (4 MiB, held on every GPU that loads the library until exit): rows above
 * 2^20 are rejected with LTB_ERR_INVALID; calls that overlap on the GPU
 * share that array and race.  The first call on a device looks up the
 * array's address; make it before any stream capture on that device. */
int ltb_row_sum_noalloc(const float* x, int64_t rows, int64_t cols, float* out,
                        void* stream);

/* ------------------------------------------------------- captured runs
 * The reference launches a multi-kernel nest's kernels one by one from the
 * host (and leaves nests that need a grid-wide sync unimplemented,
 * src/backends/cuda/cuda.cpp:726-782).  ltb_graph_create captures one run
 * of a compiled loop tree on fixed device or managed buffers -- operand
 * packing, every stage, split-K combines -- into a CUDA graph;
 * ltb_graph_run replays it with one launch, reading the buffers' current
 * contents.  scratch: caller scratch as for ltb_run_with_scratch, or NULL
 * for the compiled object's own.  Schedules changed after the capture are
 * not seen by it; the compiled object must outlive the captured run. */
typedef struct ltb_graph ltb_graph;
int ltb_graph_create(ltb_compiled* c, void* const* memory, int n, void* scratch,
                     void* stream, ltb_graph** out);
int ltb_graph_run(ltb_graph* g, int sync, void* stream);
int ltb_graph_release(ltb_graph* g);

/* ---------------------------------------------------------- autotuner
 * Replaces the reference's manual schedule search: python/ui.py:34-45
 * (benchmark a tensor's loop tree) driving the LoopTree mutations of
 * include/loop_tool/mutate.h:13-60 (split, annotate, unroll).  Here the
 * schedule space is the B200 kernels' own: per stage the grid (CTAs per SM,
 * the "parallel" annotation), the CTA size ("threaded"), the row-softmax
 * elements/threads pair and the tensor-core tile width (128 or 256).
 *
 * ltb_tune times every candidate schedule of every stage on `memory`
 * (device or managed buffers, as ltb_run), keeps the fastest, leaves the
 * outputs computed with it, records it in the process-wide schedule cache
 * and writes a report (one line per stage, in annotation vocabulary) into
 * report[len] if report is not NULL.  The cache key is a hash of the IR text
 * (which carries every size) and the compile options; ltb_compile applies a
 * cached schedule (int property "tuned" = 1).  reps: timed runs per
 * candidate. */
int ltb_tune(ltb_compiled* c, void* const* memory, int n, void* stream, int reps,
             char* report, size_t len);
/* Read or set one stage's schedule (zeros = the built-in heuristic;
 * threads in {0, 64, 128, 256, 512}; variant: family-specific).  For a
 * tensor-core contraction, variant = tile width | form: 128 / 256 row-store
 * epilogue, 129 / 257 shared-memory transposed epilogue, 130 two 128-wide
 * CTAs per SM, 131 halo image tiles with resident weights (single-segment
 * convolutions whose weights fit in shared memory; elsewhere it reads back
 * as 128), 133 the same halo tiles two to a CTA pair (M = 256, half of the
 * weights in each CTA; elsewhere 128), 258 256 x 256 tiles on CTA pairs
 * (plain operands; elsewhere 256); cta_per_sm is the raster group.  For a CUDA-core (FP32)
 * contraction, variant = 64 or 128 is the CTA tile (0: 64 when the problem
 * has at most SMs / 4 tiles of 128 x 128); both give the same bits.  For a
 * pooling reduction, variant 4 runs 4 work items per thread (else 2). */
int ltb_get_schedule(ltb_compiled* c, int stage, int* cta_per_sm, int* threads,
                     int* variant);
int ltb_set_schedule(ltb_compiled* c, int stage, int cta_per_sm, int threads,
                     int variant);
/* Store the compiled object's current schedules in the cache. */
int ltb_tune_record(ltb_compiled* c);

/* The compiled object's current launch schedule written into its loop tree
 * in the reference's annotation vocabulary (serialize() text that the
 * reference's deserialize reads, serialization.cpp:239-332; the portable
 * schedule record of the reference's IR-text format, :175-237).  For each
 * grid-stride elementwise / serial-reduction stage the outermost unsplit
 * output loop v of size S is split into v(S / (G*T), S % (G*T)),
 * v(G) "parallel", v(T) "parallel" -- G CTAs of T threads; for a tree
 * reduction the innermost unsplit reduced loop r of size R into
 * r(R / T, R % T), r(T) "parallel" -- T threads per output.  Splits keep
 * each var's visiting order, so values do not change.  ltb_compile of the
 * text pins the same choices (a "parallel" loop's iteration counts fix the
 * thread count; the autotuner leaves pinned choices alone).  Stages whose
 * choices the vocabulary cannot express (fused row kernels, tensor-core
 * tiles) keep theirs in the schedule cache (ltb_tune_save). */
int ltb_schedule_ir(ltb_compiled* c, char* buf, size_t len);
/* Cache persistence: a text file holding, per entry, the serialized IR
 * (src/core/serialization.cpp:175-237 format), the options and one
 * schedule line per stage.  Loading merges into the cache. */
int ltb_tune_save(const char* path);
int ltb_tune_load(const char* path);
int ltb_tune_clear(void);
int64_t ltb_tune_entries(void);

/* Stream synchronisation helper (cuCtxSynchronize in the reference,
 * src/backends/cuda/cuda.cpp:847-849, when stream is NULL).  Also reports
 * (LTB_ERR_TIMEOUT, once) a bounded wait that gave up in a kernel launched
 * on this stream of the current device since the stream's last
 * synchronising call: every device wait in these kernels is bounded, and
 * its timeout flag is kept per stream. */
int ltb_synchronize(void* stream);

/* Self-check of the bounded device waits, on the current device and
 * `stream`: one CTA allocates TMEM, starts a bulk copy, then waits on an
 * mbarrier that nothing ever arrives at for at most limit_cycles clock
 * cycles (1 .. 4e9; the kernels' own waits allow about 2 s).  The wait
 * gives up, raises the stream's timeout flag, lets its copy land, frees
 * the TMEM and returns; the call then reports LTB_ERR_TIMEOUT with
 * *completed = 0 and *drained = 1.  Exercises, on the GPU, the give-up path
 * every wait in the tensor-core and bulk-copy kernels takes, without a
 * fault or a hang.  No reference counterpart (the reference's kernels never
 * wait on the device). */
int ltb_check_bounded_wait(int64_t limit_cycles, void* stream, int* completed,
                           int* drained);

/* ------------------------------------------------------------- serving
 * A native continuous-batching request loop.  The reference has none: its
 * lazy frontend runs one program at a time, synchronously, allocating each
 * output (include/loop_tool/lazy.h:249-258).  The server keeps one CUDA
 * stream ("slot") per concurrent request and one device workspace per slot
 * (inputs, output and run scratch of its request, grown stream-ordered only
 * when a request needs more), admits requests in arrival order while a slot
 * is free and their bytes (ltb_io_sizes + scratch_bytes) fit the HBM budget,
 * compiles each distinct loop tree once (kernel cache keyed by IR text),
 * generates each request's inputs on the device from its seed, and runs it
 * with caller scratch (ltb_run_with_scratch), so concurrent requests share
 * nothing.  Latency is arrival to completion (the slot's event), on the
 * host's steady clock. */
#define LTB_SERVE_MAX_IO 8
typedef struct {
  int64_t rows, cols;           /* the buffer: rows x cols floats, row-major */
  int64_t true_rows, true_cols; /* the request's own top-left block; the rest
                                   is shape-bucket padding, zero in inputs */
  float scale;                  /* inputs: seeded N(0, 1) values times scale */
} ltb_block;
typedef struct {
  const char* ir_text;          /* the request's loop tree (serialize text) */
  double arrival_s;             /* arrival time from the start of the trace */
  uint64_t seed;                /* seed of its inputs */
  int n_io;                     /* inputs + outputs of the loop tree */
  ltb_block io[LTB_SERVE_MAX_IO];
  float* host_out;              /* NULL, or host memory receiving the first
                                   output's true block when the request ends */
} ltb_request;
typedef struct {
  int64_t requests, compiles, peak_inflight, peak_bytes;
  double span_s, req_per_s, p50_ms, p99_ms, mean_ms, compile_s;
} ltb_serve_stats;
typedef struct ltb_server ltb_server;
/* slots >= 1 concurrent requests, hbm_budget bytes of request buffers at
 * once, options as for ltb_compile (e.g. "precision=bf16x3"). */
int ltb_server_create(int slots, int64_t hbm_budget, const char* options, ltb_server** out);
/* Compiles every distinct loop tree of reqs[0..n) and sizes every slot's
 * workspace for the largest request (within the budget), so that serving
 * them compiles and allocates nothing; *reserved_bytes (optional) = the
 * workspace bytes held. */
int ltb_server_prepare(ltb_server* s, const ltb_request* reqs, int n, int64_t* reserved_bytes);
/* Serves reqs[0..n) against the wall clock (arrival times scaled by
 * time_scale); latency_s (optional) receives each request's latency, in
 * request order.  A request larger than the budget is an error
 * (LTB_ERR_INVALID) before anything runs. */
int ltb_server_serve(ltb_server* s, const ltb_request* reqs, int n, double time_scale,
                     ltb_serve_stats* stats, double* latency_s);
int ltb_server_release(ltb_server* s);

#ifdef __cplusplus
}
#endif

#endif /* LOOP_TOOL_B200_H_ */
