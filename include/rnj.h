/*
 * rnj.h -- C ABI of librnjgpu.so, the B200 (sm_100a) distance-estimation path of
 * rapidNJ.
 *
 * The library replaces the all-pairs distance matrix that rapidNJ builds from an
 * alignment (src/distanceCalculation/ of rapidNJ):
 *   - DNA: Jukes-Cantor and Kimura two-parameter distances,
 *   - protein: Jukes-Cantor and Kimura's protein distance (Dayhoff PAM table),
 * with the reference's packing rules, per-pair counts, transforms and
 * post-process (mirror, zero diagonal, saturated pairs -> 2 * max).
 *
 * Every entry point returns an rnj_status; on failure rnj_last_error() holds a
 * message for the calling thread.  Nothing here calls exit().
 *
 * Objects (rnj_ctx, rnj_aln, rnj_mat, rnj_batch, rnj_server) are opaque.  A context
 * owns one CUDA stream on one device and is not shared between host threads.
 * Device pointers passed in or out are plain CUDA device addresses on the
 * context's device.
 */
#ifndef RNJ_H
#define RNJ_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------------------------------------------------------- constants */

typedef enum {
  RNJ_OK = 0,
  RNJ_ERR_INVALID = 1,     /* bad argument */
  RNJ_ERR_CUDA = 2,        /* a CUDA runtime call failed */
  RNJ_ERR_NOMEM = 3,       /* device or pinned host allocation failed */
  RNJ_ERR_IO = 4,          /* file could not be read / written */
  RNJ_ERR_FORMAT = 5,      /* malformed alignment (ragged rows, < 2 sequences, ...) */
  RNJ_ERR_TIMEOUT = 6,     /* a bounded device or host wait ran out */
  RNJ_ERR_BUSY = 7,        /* admission refused (not enough free device memory) */
  RNJ_ERR_UNSUPPORTED = 8, /* option not available in this build */
  RNJ_ERR_NOTREADY = 9     /* request still running */
} rnj_status;

/* Sequence type; same values as InputType in rapidNJ src/stdinclude.h:26. */
typedef enum { RNJ_DNA = 0, RNJ_PROTEIN = 1, RNJ_UNKNOWN = 2 } rnj_type;

/* Evolution model (-a jc / -a kim, src/main.cpp:253-274). */
typedef enum { RNJ_JC = 0, RNJ_KIMURA = 1 } rnj_model;

/* Alignment flags. */
enum {
  /* Bit-string fast path, the CLI default (src/main.cpp:597).  Without it the
   * counts follow the naive estimator used by -f
   * (src/distanceCalculation/simpleDistanceCalculator.cpp:40-98). */
  RNJ_FASTDIST = 1,
  /* Reproduce the fast protein estimator's valid-site arithmetic for
   * L % 128 == 0 (bitDistanceProtein.cpp:15-16,59), which subtracts 128 extra
   * padding gaps and can wrap.  Off by default: the default counts are the
   * correct ones, equal to the naive estimator's. */
  RNJ_COMPAT_PROTEIN_WRAP = 2,
  /* Compute every (row, column) pair in row order instead of the upper triangle
   * plus mirror, as the disk-matrix driver does (KimuraDistance.cpp:308-354 with
   * dm != NULL).  Only differs for the naive DNA estimator, whose counts are
   * asymmetric. */
  RNJ_FULL_ROWS = 4,
  /* DNA on the fast path and protein (with at most 31 distinct residues) are
   * counted on the tensor cores by default (tcgen05 kind::mxf4: FP4 features in
   * {-1, 0, +1} with unit block scales, exact f32 sums).  This flag selects the
   * bit-plane popcount kernels instead: same counts, far fewer bytes of packed
   * input per site.  DNA with the -f rules always uses the popcount kernels. */
  RNJ_POPCOUNT = 8
};

typedef struct rnj_ctx rnj_ctx;
typedef struct rnj_aln rnj_aln;
typedef struct rnj_mat rnj_mat;

/* ------------------------------------------------------------------ general */

const char *rnj_version(void);
const char *rnj_last_error(void);

/* Context on CUDA device `device`.  Replaces initialiseDNA_gpu /
 * initialiseProtein_gpu of the reference's CUDA glue (KimuraDistance.cpp:17-28).
 * Device buffers come from the device's default stream-ordered memory pool;
 * creating a context sets that pool to keep freed memory for reuse (release
 * threshold UINT64_MAX). */
int rnj_ctx_create(int device, rnj_ctx **out);
int rnj_ctx_destroy(rnj_ctx *ctx);
/* The context's CUDA stream (a cudaStream_t). */
int rnj_ctx_stream(rnj_ctx *ctx, void **stream);
int rnj_ctx_synchronize(rnj_ctx *ctx);

/* Every pipeline wait in the counting kernels (a warp waiting for a copy into
 * shared memory, for the tensor cores, or for tensor memory to be read) is
 * bounded: when it runs out, the kernel stops, lets its own copies land, frees
 * its tensor memory and sets the context's device error word, and the next call
 * that waits for the GPU (rnj_ctx_synchronize, any call returning a maximum)
 * returns RNJ_ERR_TIMEOUT and clears the word.  rnj_set_wait_limit sets that
 * bound for kernels launched from now on in this process, in microseconds
 * (0: the default, 2 seconds).  No counterpart in the reference, which has no
 * device code in its build. */
int rnj_set_wait_limit(unsigned int microseconds);
/* For tests of that failure path: while `on` is non-zero, the consumer warps of
 * the single-alignment counting kernels first wait on a barrier that nothing
 * completes, so that their bounded wait runs out (after the wait limit) and the
 * call reports RNJ_ERR_TIMEOUT; nothing faults or hangs, and the context stays
 * usable.  Off by default. */
int rnj_test_wait_on_unset_flag(int on);

/* Stage timing: when on, the library records CUDA events around its kernels
 * (pack, count, transform/fix-up) on the context's stream;
 * rnj_ctx_stage_times() synchronises and returns the last call's milliseconds
 * per stage in ms[0..2]: pack, count (incl. a split-K transform), fix-up. */
int rnj_ctx_set_profiling(rnj_ctx *ctx, int on);
int rnj_ctx_stage_times(rnj_ctx *ctx, float *ms);

/* Measured device-wide throughput of the two integer pipes the counting kernels
 * run on: POPC and LOP3 operations per second (a short microbenchmark). */
int rnj_probe_int_peaks(rnj_ctx *ctx, double *popc_per_s, double *lop3_per_s);
/* FP4 tensor-pipe throughput of the context's device in flop/s: every SM issues
 * back-to-back 128 x 128 x 64 tcgen05 kind::mxf4 MMAs (the instruction the DNA
 * counting kernel uses) with operands already in shared memory.  No counterpart
 * in the reference; the roofline of the tensor-core kernel is quoted against it. */
int rnj_probe_tc_peak(rnj_ctx *ctx, double *fp4_flops_per_s);
/* Self-check of the fused epilogue's quotients on the device, against
 * correctly rounded division: the float quotients by the valid count (the
 * reference's (float)((double)num / (double)n)) for every 0 <= num <= n < 2^16,
 * and JC's (double)p / b for every float p in [0, 1] and b = 3/4, 19/20.
 * *mismatches is 0 on a sound build.  No counterpart in the reference. */
int rnj_check_quotient16(rnj_ctx *ctx, unsigned long long *mismatches);

/* Sequence type of an alignment from its first sequence: any byte >= 65 outside
 * ACGTUN/acgtun makes it protein (dataloaderFasta.hpp:54-76). */
int rnj_detect_type(const char *seq0, int L);

/* --------------------------------------------------------- alignment upload */

/* Packs n sequences of L bytes each into the device bit-plane layout.  Replaces
 * the loader's packing (encodeDNASequence / encodeProteinSequence,
 * dataloaderFasta.hpp:135-182) and storeDataDNA_gpu (KimuraDistance.cpp:19).
 * `type` RNJ_UNKNOWN detects it from seqs[0].  `flags` is RNJ_FASTDIST |
 * RNJ_COMPAT_PROTEIN_WRAP | RNJ_FULL_ROWS.  Bytes are the characters of the
 * alignment as the reference's parsers keep them (33..126). */
int rnj_aln_from_host(rnj_ctx *ctx, const char *const *seqs, int n, int L, int type,
                      int flags, rnj_aln **out);
/* Same, from one host buffer of n rows with stride ld >= L. */
int rnj_aln_from_host_buffer(rnj_ctx *ctx, const char *chars, int n, int L, size_t ld,
                             int type, int flags, rnj_aln **out);
/* Same, from a device buffer already on the context's device. */
int rnj_aln_from_device(rnj_ctx *ctx, const void *d_chars, int n, int L, size_t ld,
                        int type, int flags, rnj_aln **out);
/* From the reference loader's packed arrays (dataloader::getBitStrings /
 * getGapFilters / getBitStringsCount, dataloader.hpp:20-24): DNA 2-bit codes, 16
 * sites per uint32 LSB first, with 01-per-valid-site gap filters; protein one
 * resolved byte per site.  This is the entry the drop-in distance classes use on
 * the fast path. */
int rnj_aln_from_bitstrings(rnj_ctx *ctx, const unsigned int *const *bit_strings,
                            const unsigned int *const *gap_filters, int n, int L,
                            int bit_strings_count, int type, int flags, rnj_aln **out);
int rnj_aln_info(const rnj_aln *aln, int *n, int *L, int *type);
int rnj_aln_destroy(rnj_aln *aln);

/* ---------------------------------------------------------------- distances */

/* Full post-processed n x n float matrix on the device: the matrix that
 * JCdistance::computeDistanceMatrix (JCdistance.cpp:24-44) and
 * KimuraDistance::computeDistances (KimuraDistance.cpp:75-99) leave behind, and
 * the replacement for computeDistancesDNA2_gpu / computeDistancesProtein_gpu
 * (KimuraDistance.cpp:21,25). */
int rnj_distance(rnj_ctx *ctx, rnj_aln *aln, int model, rnj_mat **out);
/* Same into a caller-owned device buffer of n rows with stride ld (floats).
 * max_out (host, may be NULL) receives the maximum distance; reading it
 * synchronises the context's stream and reports a device timeout.  With
 * max_out NULL the call returns without waiting for the GPU: a timeout is then
 * reported by the next call on the context that waits (rnj_ctx_synchronize). */
int rnj_distance_into(rnj_ctx *ctx, rnj_aln *aln, int model, float *d_out, size_t ld,
                      float *max_out);
/* Raw per-pair counts, the DistanceEstimate::computeDistance contract
 * (DistanceEstimate.hpp:14): {ts, tv, valid} for DNA, {mismatch, 0, valid} for
 * protein, as n*n*3 uint32 on the device, written for j > i (every pair with
 * RNJ_FULL_ROWS; every other entry is set to zero).  The valid count is the
 * correct one; RNJ_COMPAT_PROTEIN_WRAP only changes distances. */
int rnj_counts_into(rnj_ctx *ctx, rnj_aln *aln, unsigned int *d_counts);
/* The distance matrix in double precision into d_out (device, n rows of stride
 * ld doubles): each pair's value is the reference's double expression before
 * its cast to distType (JCdistance.cpp:171-183, KimuraDistance.cpp:322-349),
 * evaluated in the same order with CUDA's double log; then the post-process
 * in double (KimuraDistance.cpp:366-395): saturated pairs (-1) become twice
 * the maximum of the doubles, the lower triangle mirrors the upper (full rows
 * with RNJ_FULL_ROWS), the diagonal is 0.  max_out (may be NULL) receives that
 * maximum.  Synchronous.  Scratch: the n x n x 3 counts (12 n^2 bytes), freed
 * before the call returns.  No counterpart in the reference, whose matrix is
 * float; (float) of each value is the reference's entry. */
int rnj_distance_f64(rnj_ctx *ctx, rnj_aln *aln, int model, double *d_out, size_t ld,
                     double *max_out);

int rnj_mat_info(rnj_mat *mat, int *n, float *max_distance);
int rnj_mat_device_ptr(rnj_mat *mat, float **d_ptr, size_t *ld);
/* Copies rows [row0, row0 + nrows) into host arrays rows[0..nrows) of n floats
 * each (for example rows allocated with new distType[n], which the join loops
 * later delete[]).  Uses pinned staging and `threads` host threads (<= 0: all
 * online cores) for the final copy. */
int rnj_mat_copy_rows(rnj_ctx *ctx, rnj_mat *mat, int row0, int nrows, float **rows,
                      int threads);
int rnj_mat_destroy(rnj_mat *mat);

/* Distances for callers that cannot allocate device memory: a process that owns
 * the whole GPU through its own memory pool, or that forbids cudaMalloc because
 * it synchronises the device.  No counterpart in the reference.  Same result as
 * rnj_distance_into, computed on the caller's `stream` (a cudaStream_t; NULL =
 * legacy default) from device bytes d_chars (n rows, stride ld) into d_out (n
 * rows, stride ld_out floats).  type must be RNJ_DNA or RNJ_PROTEIN.  No context
 * is needed and nothing is allocated: every intermediate buffer lives in one
 * 16 MiB array built into the library, which each GPU that loads the library
 * holds until the process exits.  Limits: the packed alignment must fit that
 * array (about n * L * 0.375 bytes for DNA, 0.5 with -f rules, 1 for protein,
 * n rounded up to 128 and L to 256) and L <= 65280; larger inputs return
 * RNJ_ERR_INVALID with the size needed.  All calls share the array and keep the
 * last call's contents (each call clears what must start at zero): calls whose
 * work overlaps on the GPU race, so issue them one after another on one stream.
 * The first call on a device looks up the array's device address and loads
 * the kernels the entry point launches (under CUDA's lazy module loading a
 * kernel's first launch would otherwise take device memory for its code); make
 * it before any stream capture.  The call returns once the GPU has finished its
 * work (it synchronises `stream`), so that a device timeout is reported in its
 * return value (RNJ_ERR_TIMEOUT) whether or not max_out is given; on a stream
 * that is being captured it returns RNJ_ERR_UNSUPPORTED before doing anything.
 * max_out (host, may be NULL) receives the maximum distance. */
int rnj_distance_noalloc(const void *d_chars, int n, int L, size_t ld, int type, int model,
                         int flags, float *d_out, size_t ld_out, void *stream, float *max_out);

/* ------------------------------------------------- matrices beyond device memory */

/* Receives rows [row0, row0 + nrows) of the distance matrix, row k at
 * rows + k * ld (page-locked host memory, valid during the call).  Returns 0 to
 * go on, non-zero to stop the computation (the call then fails). */
typedef int (*rnj_rows_fn)(void *user, int row0, int nrows, const float *rows, size_t ld);

/* The distance matrix of an alignment whose n x n floats need not fit in device
 * memory: the rows are computed in bands of band_rows (rounded up to 128; 0:
 * two bands of at most 512 MiB) with device buffers for two bands only, and
 * handed to fn in row order while the next band computes.  Each row is complete
 * (j = 0 .. n - 1, every ordered pair counted, as rapidNJ's disk-matrix drivers
 * compute them, KimuraDistance.cpp:308-354 / JCdistance.cpp:160-195 with
 * dm != NULL), with 0 on the diagonal and -1 for saturated pairs: the rows
 * those drivers pass to diskMatrix::writeArray (diskMatrix.cpp:96-117).  When
 * the call returns, *max_out holds the maximum distance and *saturated_out
 * (both may be NULL) is 1 if any pair saturated; the caller's post-process then
 * replaces every -1 by 2 * max (KimuraDistance.cpp:366-395,
 * JCdistance.cpp:201-230).  Alignments of at most 65535 columns (tensor-core
 * layouts) or 65280 (bit planes).  Device memory: the packed alignment, two
 * bands of band_rows x n floats, one int per 128 x 128 tile of the full square. */
int rnj_distance_rows(rnj_ctx *ctx, rnj_aln *aln, int model, int band_rows, rnj_rows_fn fn,
                      void *user, float *max_out, int *saturated_out);

/* Free and total memory of the context's device, in bytes (cudaMemGetInfo). */
int rnj_ctx_memory(rnj_ctx *ctx, size_t *free_bytes, size_t *total_bytes);

/* One call, host in / host out: pack, distances, copy into out (n*n floats,
 * row-major).  max_out may be NULL.  This is what JCdistance::computeDistanceMatrix
 * (JCdistance.cpp:24-44) and KimuraDistance::computeDistances
 * (KimuraDistance.cpp:75-99) produce, from the loader's sequences to the filled
 * matrix.  For DNA and protein on the tensor-core kernel with a page-locked `out`
 * and n above 1408 (12 tile rows; below that one upload, one launch sequence and
 * one download are faster), the call is streamed: bands of rows are computed
 * last band first, and each band's finished rows and columns are copied to `out`
 * while later bands are uploaded and computed (the n*n*4-byte download then
 * bounds the call). */
int rnj_distance_matrix_host(rnj_ctx *ctx, const char *chars, int n, int L, size_t ld,
                             int type, int model, int flags, float *out, float *max_out);
/* The same with the band height of the streamed form in 128-row tiles:
 * 0 = the library's choice (not streamed below 12 tile rows), > 0 = that many
 * tile rows per band (streamed at any size), < 0 = not streamed (upload,
 * compute, then one download). */
int rnj_distance_matrix_host_ex(rnj_ctx *ctx, const char *chars, int n, int L, size_t ld,
                                int type, int model, int flags, int band_tiles, float *out,
                                float *max_out);

/* ------------------------------------------------------------------ batches */

/* Many alignments computed together.  The triangle tiles of every alignment
 * added form one device work list, ordered by decreasing cost, that one
 * persistent launch per kernel family consumes (the tensor-core kernel for DNA,
 * the bit-plane kernel for protein and -f alignments), followed by the
 * saturation fix-up; the launch sequence is captured once, at creation, in a
 * CUDA graph, and a run only uploads the descriptors and work lists the graph
 * reads.  For a stream of alignments this replaces one driver call per
 * alignment (JCdistance / KimuraDistance per input, or per bootstrap replicate
 * of main.cpp:519-532).  Capacities bound the alignments and the total tiles
 * (128 x 128 pairs each, (ceil(n/128)+1)*ceil(n/128)/2 per alignment).  The
 * alignments added must stay alive until the run has completed.  Alignments
 * longer than 65535 columns (tensor cores) or 65280 (bit planes) are not
 * batched (use rnj_distance). */
typedef struct rnj_batch rnj_batch;
int rnj_batch_create(rnj_ctx *ctx, int max_alignments, long long max_tiles, rnj_batch **out);
/* Adds an alignment; d_out NULL lets the batch allocate the n x n output.  The
 * slot index identifies the alignment in this batch. */
int rnj_batch_add(rnj_batch *batch, rnj_aln *aln, int model, float *d_out, size_t ld, int *slot);
/* Packs and adds `count` alignments already on the device (d_chars[k]: n[k] rows
 * of stride ld[k], L[k] columns, type[k] RNJ_DNA or RNJ_PROTEIN, model[k]) in one
 * call: the residue alphabets of all protein alignments are scanned with a
 * single synchronisation.  The batch owns these packed alignments (freed by
 * rnj_batch_clear / _destroy).  d_out / ld_out may be NULL (batch-allocated
 * outputs); slots (may be NULL) receives the slot of each alignment. */
int rnj_batch_add_many(rnj_batch *batch, int count, const void *const *d_chars, const int *n,
                       const int *L, const size_t *ld, const int *type, const int *model,
                       int flags, float *const *d_out, const size_t *ld_out, int *slots);
/* Runs the batch asynchronously after the work already queued on the context
 * stream; later work on that stream sees the results. */
int rnj_batch_run(rnj_batch *batch);
int rnj_batch_synchronize(rnj_batch *batch);
/* Non-blocking: *done = 1 once the last run has completed on the device. */
int rnj_batch_poll(rnj_batch *batch, int *done);
/* The output of a slot (device pointer and stride); max_out (may be NULL)
 * waits for the run and reads the slot's maximum distance. */
int rnj_batch_output(rnj_batch *batch, int slot, float **d_out, size_t *ld, float *max_out);
/* Moves a batch-allocated output into a matrix handle (for rnj_mat_copy_rows). */
int rnj_batch_take(rnj_batch *batch, int slot, rnj_mat **out);
int rnj_batch_size(rnj_batch *batch, int *alignments, long long *tiles);
/* The launch shape of the last run: the tensor-core ring depth it ran with
 * (the tuned depth of the bucket holding most of its work) and how many of its
 * alignments had a tuned entry (each one's tile-order band comes from it).
 * Either pointer may be NULL. */
int rnj_batch_tuning(rnj_batch *batch, int *ring_depth, int *tuned_alignments);
/* Forgets the alignments (frees outputs still owned by the batch); the graph stays. */
int rnj_batch_clear(rnj_batch *batch);
int rnj_batch_destroy(rnj_batch *batch);

/* Bootstrap replicates on the device: the loop of main.cpp:519-532 with the
 * column resampling of dataloader::sample_fast_dist (dataloader.cpp:16-58).
 * Replicate r is the alignment whose column k is column cols[r * L + k] of the
 * original (device bytes d_chars, n rows of stride ld); rapidNJ draws these
 * columns as rand() % L after srand(0), so a caller that draws them the same
 * way gets its replicates.  The replicates are gathered on the device and
 * computed as batches; d_out[r] (device, n rows of stride ld_out floats)
 * receives replicate r's post-processed matrix and max_out[r] (host, may be
 * NULL) its maximum distance.  n <= 32,640.  Returns when all are done. */
int rnj_bootstrap(rnj_ctx *ctx, const void *d_chars, int n, int L, size_t ld, int type,
                  int model, int flags, int R, const int *cols, float *const *d_out,
                  size_t ld_out, float *max_out);

/* ------------------------------------------------------------------ serving */

/* Continuous batching of distance requests.  Clients submit host alignments
 * from any thread; a scheduler thread of the server (with its own context on
 * `device`) admits requests first come, first served while the device memory
 * they need (bytes, packed operands, output) fits `memory_budget` (0: 60 % of
 * the free memory at creation), at most `max_batch` per scheduling pass,
 * uploads and packs them, and appends their tiles to a live work list that one
 * persistent kernel consumes while it runs: a request that arrives while
 * others compute joins the running launch, and completes on its own as soon
 * as its last tile is done (the kernel then applies its saturation fix-up and
 * flags it complete to the host).  Requests the tensor-core kernel cannot take
 * (protein alphabets above 31 residues, the -f rules, RNJ_POPCOUNT, more than
 * 65,535 columns) run as plain calls.  Packed inputs are freed when a request
 * completes; its output matrix stays on the device until the client takes it.
 * No counterpart in the reference (which computes one matrix per process run). */
typedef struct rnj_server rnj_server;
enum { RNJ_REQ_QUEUED = 0, RNJ_REQ_RUNNING = 1, RNJ_REQ_DONE = 2, RNJ_REQ_FAILED = 3 };
int rnj_server_create(int device, size_t memory_budget, int max_batch, rnj_server **out);
/* chars: n rows of stride ld; the bytes are copied before the call returns. */
int rnj_server_submit(rnj_server *server, const char *chars, int n, int L, size_t ld, int type,
                      int model, int flags, uint64_t *id);
int rnj_server_poll(rnj_server *server, uint64_t id, int *state);
int rnj_server_wait(rnj_server *server, uint64_t id, int timeout_ms);
/* Hands the finished matrix to the caller.  `owner` (a context of the caller on
 * the same device) becomes the matrix's context: it is read and freed on that
 * context's stream and outlives the server; pass it to rnj_mat_copy_rows too.
 * latency_ms (may be NULL) is the time from submit to the matrix complete on
 * the device. */
int rnj_server_result(rnj_server *server, uint64_t id, rnj_ctx *owner, rnj_mat **out,
                      double *latency_ms);
/* Completed requests, their pair-columns, the seconds from the first submit to
 * the last completion, and the device bytes the server currently holds. */
int rnj_server_stats(rnj_server *server, uint64_t *completed, double *pair_columns,
                     double *seconds, size_t *bytes_in_use);
int rnj_server_destroy(rnj_server *server);

/* ------------------------------------------------------------ shards */

/* One alignment over several GPUs, one process (and context) per GPU.  The
 * triangle tiles (128 x 128 pairs; every tile with RNJ_FULL_ROWS -f alignments)
 * are split into `nshards` contiguous ranges of equal tile count, in row-major
 * order of the upper triangle; shard s computes range s into its own n x n
 * device buffer (each tile and its mirror).  The post-process needs the maximum
 * over the whole matrix before any saturated pair is replaced
 * (KimuraDistance.cpp:366-395, JCdistance.cpp:201-230), so a shard runs in two
 * steps around one exchange, which the caller makes with its own collective:
 *   rnj_shard_run(shard, &local)         counts + transform, local maximum
 *   global = max over shards of local    (one float, e.g. an NCCL all-reduce)
 *   rnj_shard_finish(shard, global)      saturated pairs -> 2 * global
 * Every shard holds the whole packed alignment (it is small next to the
 * matrix).  No counterpart in the reference, which runs on one host. */
typedef struct rnj_shard rnj_shard;
/* Number of tiles of an n-sequence alignment and the range [tile0, tile1) of
 * shard `shard` of `nshards`.  Host arithmetic only. */
int rnj_shard_tiles(int n, int full_rows, int shard, int nshards, long long *tile0,
                    long long *tile1, long long *ntiles);
/* Row and column tile of linear tile index `tile` (row-major upper triangle, or
 * row-major full square with full_rows).  Host arithmetic only. */
int rnj_tile_coords(int n, int full_rows, long long tile, int *tile_row, int *tile_col);
/* d_out: n rows of stride ld floats on the context's device (NULL: allocated by
 * the shard and freed with it).  The alignment must outlive the shard. */
int rnj_shard_create(rnj_ctx *ctx, rnj_aln *aln, int model, int shard, int nshards,
                     float *d_out, size_t ld, rnj_shard **out);
/* Computes this shard's tiles (saturated pairs hold -1) and returns their
 * maximum distance (synchronises the context's stream). */
int rnj_shard_run(rnj_shard *shard, float *local_max);
/* Replaces the shard's saturated pairs with 2 * global_max and synchronises. */
int rnj_shard_finish(rnj_shard *shard, float global_max);
/* The shard's output (device pointer and stride). */
int rnj_shard_output(rnj_shard *shard, float **d_out, size_t *ld);
/* Copies the shard's own tiles (upper-triangle blocks; every block with
 * RNJ_FULL_ROWS) into the host matrix `host` (n rows of stride host_ld floats),
 * one 2-D copy per tile row; entries of other shards are not touched.  Returns
 * the bytes copied in *bytes (may be NULL). */
int rnj_shard_copy_tiles(rnj_shard *shard, float *host, size_t host_ld, size_t *bytes);
int rnj_shard_destroy(rnj_shard *shard);

/* ------------------------------------------------------- alignment files */

/* A parsed multiple alignment on the host: names and n*L bytes (row-major). */
typedef struct rnj_msa rnj_msa;

/* Reads a single-line FASTA ("fa") or Stockholm ("sth") alignment with the
 * reference loaders' rules (dataloaderFasta.hpp:78-133,201-276;
 * dataloaderStockholm.hpp:79-120,185-307): characters <= 32 are dropped from
 * sequence lines, every sequence must have the first one's length.  format
 * NULL picks by file extension as main.cpp:646-683 does. */
int rnj_msa_read(const char *path, const char *format, rnj_msa **out);
int rnj_msa_info(const rnj_msa *msa, int *n, int *L, int *detected_type);
const char *rnj_msa_name(const rnj_msa *msa, int i);
const char *rnj_msa_chars(const rnj_msa *msa);
int rnj_msa_destroy(rnj_msa *msa);

/* Reads an alignment file onto the device of ctx (the input side of
 * dataloaderFasta::parseData, dataloaderFasta.hpp:78-133,201-276, run on the
 * GPU): the file's bytes are read by several host threads into page-locked
 * memory and copied once; kernels find the lines, count each line's kept bytes
 * (> 32), assign lines to sequences, check the lengths and compact the bytes
 * into an n x L array on the device.  Names and results are the host reader's
 * (rnj_msa_read) for every input; FASTA files whose names end on a control byte
 * other than a final '\r', that hold data before the first name or names
 * without data, and Stockholm files, are parsed by the host rules and then
 * copied to the device.  rnj_msa_info / _name work as for rnj_msa_read;
 * rnj_msa_chars copies the bytes to the host on first use. */
int rnj_msa_read_device(rnj_ctx *ctx, const char *path, const char *format, rnj_msa **out);
/* The device bytes of an alignment read by rnj_msa_read_device (n rows of
 * stride *ld = L bytes); RNJ_ERR_INVALID for one read on the host. */
int rnj_msa_device_chars(const rnj_msa *msa, const void **d_chars, size_t *ld);

/* The "-o m" text of an n x n DEVICE matrix (rows of stride ld floats), as
 * rnj_write_matrix_text writes it (byte-identical), formatted on the device: the
 * six-decimal digits of a float are computed exactly (v * 10^6 is exact in
 * double; rounded to an integer with ties to even, as the C library prints),
 * rows are formatted in bands of up to 64 MB and written while the next band is
 * formatted.  Rows holding values of 8e9 or more in magnitude, infinities or
 * NaNs are printed by the host.  path NULL writes to stdout. */
int rnj_write_matrix_text_device(rnj_ctx *ctx, const char *path, const char *const *names,
                                 const float *d_matrix, size_t ld, int n);

/* Writes the "-o m" text matrix of main.cpp:212-221 ("\t<n>", then per row the
 * name, a tab and n values printed with six fixed decimals, each followed by a
 * space).  rows[i] are n floats; path NULL writes to stdout. */
int rnj_write_matrix_text(const char *path, const char *const *names, const float *const *rows,
                          int n, int threads);

/* ---------------------------------------------------------------- autotuner */

/* Launch parameters of one bucket of inputs: the alphabet (DNA or protein),
 * the counting rules (RNJ_FASTDIST or not), floor(log2 n) and floor(log2 L).
 * No counterpart in the reference (its CPU code has nothing to tune).  The
 * tile edge itself is fixed at 128 pairs: the tensor-core MMA is 128 rows
 * (M = 128) and three 128-column f32 accumulators fill the 512 columns of
 * tensor memory with the scale factors, and every path (transform, fix-up,
 * streamed, sharded, batched, row-band) shares that tile order.  What varies
 * is how the tiles are scheduled, how the columns are split, which epilogue
 * form runs and how deep the shared-memory rings of staged K blocks are.
 * Zero fields mean the default. */
typedef struct rnj_tune_params {
  int dna_kernel;      /* DNA fast rules and protein: 0 tensor cores, 1 bit-plane popcount */
  int ksplit;          /* bit-plane kernel: columns split over this many CTAs per tile */
  int tile_band;       /* tensor-core kernel: tile-order band height in tile rows (0 = 12) */
  int transform_ctas;  /* tensor-core transform: resident CTAs per SM, 1..5 (0 = 5) */
  int stream_band;     /* rnj_distance_matrix_host: band height in tile rows (0 = automatic) */
  int tc_epilogue;     /* tensor cores: 0 the exact transform in the counting kernel's own
                          epilogue warps (one launch), 1 packed counts and a separate
                          transform kernel at higher occupancy */
  int tc_stages;       /* tensor cores: shared-memory ring depth in 256-column K blocks,
                          2..6 fused, 2..7 two-kernel (0 = the deepest) */
  int pop_stages;      /* bit-plane kernel: ring depth in 256-site K blocks, raised to the
                          3 (DNA, 2-bit codes) or 2 (5- and 7-bit codes) its distance
                          staging needs; 0 = the deepest, 4 (DNA, 2-bit) or 3 */
  float ms;            /* the tuned configuration's time for the measured shape (output) */
} rnj_tune_params;

/* Times the candidate configurations of the bucket of (n, L, type, flags) on a
 * seeded synthetic alignment of exactly n x L (related sequences with gaps) on
 * the context's device, through the same calls as rnj_distance_into and
 * rnj_distance_matrix_host, and stores the fastest in the process-wide table
 * that every later call of that bucket uses.  Every candidate computes the same
 * distances; only the time differs.  If the environment variable
 * RNJ_TUNE_CACHE names a file, the table is read from it on first use and
 * written back after each rnj_tune; otherwise the table shipped beside the
 * library (tune_b200.txt in the directory of librnjgpu.so, measured on a B200
 * by rapidnj_b200/make_tune_table.py) is read on first use, unless
 * RNJ_NO_TUNE_TABLE is set.  out (may be NULL) receives the choice. */
int rnj_tune(rnj_ctx *ctx, int n, int L, int type, int flags, rnj_tune_params *out);
/* The stored entry of the bucket (RNJ_ERR_NOTREADY if there is none). */
int rnj_tune_get(int n, int L, int type, int flags, rnj_tune_params *out);
/* Stores an entry for the bucket (fields validated; RNJ_ERR_INVALID if out of range). */
int rnj_tune_set(int n, int L, int type, int flags, const rnj_tune_params *params);
/* Empties the table. */
int rnj_tune_clear(void);
/* Writes / reads the table as text, one bucket per line (reading merges). */
int rnj_tune_save(const char *path);
int rnj_tune_load(const char *path);

/* ---------------------------------------------------------------------------
 * Neighbour-joining set-up over a finished distance matrix (the O(n^2) passes
 * rapidNJ makes before its first join: rapidNJ::initialize, rapidNJ.cpp:94-141;
 * rapidNJMem::initialize, rapidNJMem.cpp:92-135; the zero scan of
 * rdDataInitialiser::processRow, rdDataInitialiser.cpp:174-189).
 * ------------------------------------------------------------------------- */

/* One entry of a sorted row: the reference's cluster_pair (cluster_pair.h:4-11),
 * same layout (id, then distance). */
typedef struct rnj_cluster_pair {
  unsigned int id;
  float distance;
} rnj_cluster_pair;

/* Outputs of rnj_nj_init; every pointer may be NULL (that output is skipped).
 * Host arrays hold n entries unless stated. */
typedef struct rnj_nj_data {
  /* separationsums: row i summed in float, column 0 first (rapidNJ.cpp:107-110). */
  float *separation_sums;
  /* separations: separation_sums[i] / (n - 2) in float (rapidNJ.cpp:111). */
  float *separations;
  /* maxRowSeparations: the largest separation of the rows before i, FLT_MIN for
   * row 0 (rapidNJ.cpp:113-118); max_separation (1 float) the largest of all. */
  float *max_row_separations;
  float *max_separation;
  /* possibleRedundantRows: 1 when the row holds a zero off the diagonal. */
  short *possible_redundant;
  /* Redundant rows (rapidNJ.cpp:121-131, handleRedundancy :156-167): row j is
   * redundant when an equal row (float ==, every column) of higher index exists;
   * it is mapped to the highest such row, its master.  index_to_id: i, or -1 for
   * a redundant row; redundant_to_master: the master, or i; redundant_count: the
   * rows of a master's class (itself included), else 1.  A master's redundantMap
   * list holds its class's other rows in descending order. */
  int *index_to_id;
  int *redundant_to_master;
  int *redundant_count;
  /* Sorted rows (buildSortedRow, rapidNJ.cpp:134-154; rapidNJMem.cpp:138-153), on
   * the DEVICE: row i (stride sorted_ld entries) receives the non-redundant j < i
   * as (j, matrix[i][j]) by ascending distance, equal distances by ascending j
   * (std::sort leaves their order unspecified); at most sorted_cap entries when
   * sorted_cap > 0 (rapidNJMem's sortedMatrixSize), all of them when <= 0.
   * row_lengths (host) receives the entries written (0 for redundant rows). */
  rnj_cluster_pair *sorted;
  size_t sorted_ld;
  int sorted_cap;
  int *row_lengths;
} rnj_nj_data;

/* The NJ set-up of the float n x n matrix d_matrix (device, stride ld floats),
 * as produced by this library (zero diagonal; RNJ_ERR_INVALID otherwise).  One
 * pass over the matrix computes the separation sums in the reference's order,
 * the zero scan and a hash of every row; rows of equal hash are compared in
 * full; the sorted rows are sorted per row on the device.  Returns when done. */
int rnj_nj_init(rnj_ctx *ctx, const float *d_matrix, int n, size_t ld, rnj_nj_data *out);

#ifdef __cplusplus
}
#endif
#endif /* RNJ_H */
