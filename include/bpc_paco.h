/*
 * bpc_paco.h -- C ABI of the B200 (sm_100a) BPC-PaCo codec.
 *
 * Drop-in for the host call surface of PabloEnfedaque/CUDA_BPC-PaCo: the same
 * entry points source/main_example.cu calls (CUDA_BPC, load_LUTs), the same
 * buffers (raster int32 DWT coefficients; an X*Y-int stream of codeblock-major
 * slots: slot[0] = MSB, slot[1..n] = 16-bit codewords in reservation order,
 * the rest -1), the same LUT text format and a bit-identical bitstream.
 *
 * Plain C types only (pointers, ints); `stream` arguments are cudaStream_t
 * passed as void*.  All functions are thread-compatible, not thread-safe:
 * serialise calls that share a LUT or the drop-in mode.
 */
#ifndef BPC_PACO_H
#define BPC_PACO_H

#ifdef __cplusplus
extern "C" {
#endif

/* Direction: the reference's enum BPC {CODE, DECODE} (source/common.h:8-11). */
enum { BPC_CODE = 0, BPC_DECODE = 1 };

/* Return values.  0 = success.  Negative = the call failed and did nothing
 * useful.  Positive = the call ran; the value is the OR of per-codeblock
 * conditions (the outputs of the affected codeblocks are defined but differ
 * from what the reference would produce, whose behaviour there is undefined):
 *   SLOT_OVERFLOW  more codewords than the slot holds (4095 for 64x64); the
 *                  excess is dropped instead of spilling into the next slot;
 *   BAD_STREAM     a slot whose MSB word is outside 0..32 (decoded as zeros);
 *   INPUT_RANGE    a coefficient with |x| >= 2^28 (flag bits would collide);
 *   LUT_RANGE      a LUT entry outside 0..255 (read as 0). */
#define BPC_OK 0
#define BPC_ERR_ARG (-1)
#define BPC_ERR_CUDA (-2)
#define BPC_ERR_FILE (-3)
#define BPC_ERR_PARSE (-4)
#define BPC_ERR_NOMEM (-5)
#define BPC_ERR_TOO_LARGE (-6) /* image larger than bpc_encode_compact_noalloc's fixed scratch, or a
                                  server request larger than the server's whole memory budget */
#define BPC_ERR_CANCELLED (-7) /* server request withdrawn by bpc_server_cancel before it ran */
#define BPC_ST_SLOT_OVERFLOW 1
#define BPC_ST_BAD_STREAM 2
#define BPC_ST_INPUT_RANGE 4
#define BPC_ST_LUT_RANGE 8

/* ---------------------------------------------------------------------------
 * Drop-in entry points
 * ------------------------------------------------------------------------- */

/* Replaces CUDA_BPC, source/BPC_PaCo.cu:1305-1325 (declared at
 * source/main_example.cu:8).  Direction BPC_CODE: HData holds HDSize_X x
 * HDSize_Y raster coefficients and is overwritten with the slot stream;
 * BPC_DECODE: the reverse.  LUT is a device pointer from load_LUTs and, as in
 * the reference (:1300), this call frees it.  Synchronous.  The coding mode
 * (passes, DWT levels, codeblock size) is the one set with bpc_set_mode,
 * replacing the reference's -DCPASS_3 / -DDWT_LEVELS / -DCBLOCK_LENGTH.
 * Errors are reported on stderr and kept for bpc_last_status(); unlike the
 * reference (common.cu:3-9) it never calls exit(). */
void CUDA_BPC(int Direction, int *HData, int HDSize_X, int HDSize_Y, int *LUT);

/* Replaces load_LUTs, source/main_example.cu:219-448: parses ref.txt,
 * sig.txt, sign.txt (+ cp_sig.txt, cp_sign.txt in 3-pass mode) from `folder`
 * (a prefix, so it normally ends in '/') with the reference's rules and
 * uploads the array to a new device buffer stored in *LUT (NULL on error). */
void load_LUTs(int **LUT, const char *folder);

/* Mode for CUDA_BPC / load_LUTs: passes 2 or 3 (CPASS_3 = 0 / 1), DWT levels
 * >= 1, codeblock size 64 (the reference) or 32.  Default 2, 5, 64. */
int bpc_set_mode(int passes, int dwt_levels, int cb_size);
int bpc_get_mode(int *passes, int *dwt_levels, int *cb_size);

/* Status of the last drop-in call (CUDA_BPC / load_LUTs) on this process. */
int bpc_last_status(void);
const char *bpc_status_string(int status);

/* ---------------------------------------------------------------------------
 * Status-returning variants
 * ------------------------------------------------------------------------- */

/* load_LUTs into host memory.  With out == NULL only *n_entries is set. */
int bpc_load_luts_host(const char *folder, int passes, int levels, int *out, int capacity, int *n_entries);

/* load_LUTs into a new device buffer (free with bpc_lut_free). */
int bpc_load_luts(const char *folder, int passes, int levels, int **d_lut, int *n_entries);
int bpc_lut_free(int *d_lut);

/* CUDA_BPC with explicit mode and LUT length, returning the status; does not
 * free the LUT.  hdata is host memory (pinned memory is fastest). */
int bpc_code_host(int direction, int *hdata, int X, int Y, const int *d_lut, int lut_n, int passes, int levels,
                  int cb_size);

/* Copy/compute pipeline of the host-buffer calls (CUDA_BPC, bpc_code_host):
 * the image is cut into bands of codeblock rows of at least band_cbs
 * codeblocks, at most max_bands of them at the steady length, each band's copy
 * in, kernel and copy out queued round-robin on `streams` (1..16) CUDA
 * streams; with ramp (0..8) > 0 the first and last `ramp` bands halve in
 * length towards both ends of the image.  Affects the speed only; the output
 * is the same for every setting.  bpc_host_band_rows returns the number of
 * bands for an X x Y image and writes the first codeblock row of each (up to
 * `capacity`) to `starts` (may be NULL). */
int bpc_set_host_pipeline(int band_cbs, int max_bands, int streams, int ramp);
int bpc_get_host_pipeline(int *band_cbs, int *max_bands, int *streams, int *ramp);
int bpc_host_band_rows(int X, int Y, int cb_size, int *starts, int capacity);

/* ---------------------------------------------------------------------------
 * Device-pointer entry points: stream-ordered, no allocation, no host sync.
 *
 * Alignment: the kernels read coefficients with 8-byte loads and slot streams
 * with 16-byte loads, so every device input that is a coefficient image
 * (encode, LUT statistics, batch encode, server encode requests) must be
 * 8-byte aligned and every slot-stream input (decode, server decode requests)
 * 16-byte aligned; other pointers are refused with BPC_ERR_ARG before anything
 * is launched.  cudaMalloc'd buffers, and offsets into them by whole
 * codeblock rows, always qualify.
 * ------------------------------------------------------------------------- */

/* Encode X x Y raster coefficients (device) into the slot stream (device,
 * X*Y ints).  X and Y must be multiples of cb_size.  d_status (device int,
 * may be NULL) receives the OR of BPC_ST_* bits (the caller zeroes it);
 * d_counts (device, one int per codeblock, may be NULL) receives the number
 * of codewords of each codeblock.  grid = 0 launches one CTA per 4
 * codeblocks; grid > 0 launches that many persistent CTAs. */
int bpc_encode_device(const int *d_coeffs, int *d_stream, int X, int Y, const int *d_lut, int lut_n, int passes,
                      int levels, int cb_size, int *d_status, int *d_counts, int grid, void *stream);

/* Decode the slot stream (device) into raster coefficients (device). */
int bpc_decode_device(const int *d_stream, int *d_coeffs, int X, int Y, const int *d_lut, int lut_n, int passes,
                      int levels, int cb_size, int *d_status, int *d_counts, int grid, void *stream);

/* The same calls with a work order: for images of more than two waves of
 * warps (above about 4,700 codeblocks for the encoder, 8,300 for the decoder
 * on a 148-SM B200) the call first sorts the codeblocks by expected work,
 * heaviest first (decoder: slot words in use and bitplanes; encoder: bitplanes
 * coded, from one read of the coefficients), so that the warps of a CTA finish
 * together and the last wave is short.  A decode of 64x64 codeblocks between
 * half a wave and two waves (about 2,100 to 8,300 codeblocks, e.g. 4096x4096)
 * is sorted the same way and then isolated: its 24 heaviest codeblocks run on
 * six SMs of their own, the rest on the other SMs as a programmatic dependent
 * launch that starts once those are resident.  Outputs are identical to the
 * calls above.  d_sched is the caller's device scratch of
 * bpc_sched_ints(X, Y, cb_size) ints (8 bytes per 64x64 codeblock plus 16),
 * reusable once the call's stream has passed it; still no allocation and no
 * host sync. */
long long bpc_sched_ints(int X, int Y, int cb_size);
int bpc_encode_device_sched(const int *d_coeffs, int *d_stream, int X, int Y, const int *d_lut, int lut_n, int passes,
                            int levels, int cb_size, int *d_status, int *d_counts, int *d_sched, void *stream);
int bpc_decode_device_sched(const int *d_stream, int *d_coeffs, int X, int Y, const int *d_lut, int lut_n, int passes,
                            int levels, int cb_size, int *d_status, int *d_counts, int *d_sched, void *stream);

/* ---------------------------------------------------------------------------
 * Batched persistent coding (no counterpart in the reference, which codes one
 * image per call): many images of mixed size, DWT levels, pass count and
 * codeblock size, one persistent kernel per (passes, codeblock size) class fed
 * from a device work queue, the whole call captured in a CUDA graph.
 * Output is the compact container: codeblock g (images in order, codeblocks in
 * raster order) occupies compact[offsets[g] .. offsets[g+1]) = MSB word then
 * its codewords; offsets has codeblocks + 1 entries.  The compact container
 * needs at most bpc_batch_words() ints.
 * ------------------------------------------------------------------------- */
int bpc_batch_create(int n_images, const int *X, const int *Y, const int *levels, const int *passes,
                     const int *cb_size, const int *const *d_luts, const int *lut_n, void **batch);
long long bpc_batch_codeblocks(const void *batch);
long long bpc_batch_words(const void *batch);
int bpc_batch_encode(void *batch, const int *const *d_coeffs, int *d_compact, long long *d_offsets, int *d_status,
                     void *stream);
int bpc_batch_decode(void *batch, const int *d_compact, const long long *d_offsets, int *const *d_coeffs,
                     int *d_status, void *stream);
/* Schedule: CTAs per SM for the encoder (1..4) and decoder (1..7), codeblocks
 * per work item, CUDA graph on/off.  bpc_batch_tune times the candidates on the
 * given buffers and keeps the fastest. */
int bpc_batch_set_schedule(void *batch, int ctas_per_sm_enc, int ctas_per_sm_dec, int cbs_per_item, int use_graph);
int bpc_batch_get_schedule(const void *batch, int *ctas_per_sm_enc, int *ctas_per_sm_dec, int *cbs_per_item,
                           int *use_graph);
/* Further schedule dimensions, per direction: warps per CTA of the persistent
 * kernels (2, 4 or 8; CTAs per SM times warps per CTA may not exceed 16 for the
 * encoder and 28 for the decoder, and bpc_batch_set_tuning lowers the CTAs per
 * SM to fit); the order in which the device queue hands out work items (0 =
 * coarse subbands first, fixed at creation; 1 = sorted by expected cost on the
 * GPU before every call: decoder container words + 128 per bitplane from the
 * offsets and MSB words, encoder bitplanes from one extra read of the
 * coefficients); and whether the kernels of the (passes, codeblock size)
 * classes run concurrently on forked streams (0) or one after another (1).
 * Outputs never depend on any schedule setting. */
int bpc_batch_set_tuning(void *batch, int warps_per_cta_enc, int warps_per_cta_dec, int cost_order_enc,
                         int cost_order_dec, int classes_in_sequence_enc, int classes_in_sequence_dec);
int bpc_batch_get_tuning(const void *batch, int *warps_per_cta_enc, int *warps_per_cta_dec, int *cost_order_enc,
                         int *cost_order_dec, int *classes_in_sequence_enc, int *classes_in_sequence_dec);
int bpc_batch_tune(void *batch, const int *const *d_coeffs, int *d_compact, long long *d_offsets, int *const *d_out,
                   void *stream, double *best_us);
int bpc_batch_destroy(void *batch);

/* One-image encode into the compact container that allocates no memory.  No
 * counterpart in the reference.  For callers that may not call cudaMalloc while
 * they code: an application whose device memory is already handed to its own
 * pool, a latency-critical stream an allocation would stall, a plugin its host
 * only gives device pointers.  The scratch this encode needs (slot stream,
 * per-codeblock counts and sizes, prefix-scan workspace) lives in one fixed
 * 16.1 MiB device array inside the library, held by every GPU that loads this
 * code until the process exits.  Limit: X*Y <= 2048*2048 coefficients, else
 * BPC_ERR_TOO_LARGE.  Output as bpc_batch_encode for a one-image batch:
 * d_compact (at most X*Y ints) and d_offsets (codeblocks + 1 entries).  The
 * first call on each device looks the array's device address up; make that
 * call before any stream capture.  The address is kept per device and CUDA
 * context: after cudaDeviceReset the next call sees a new context and looks it
 * up again (so that call is a first call too).  All calls share the array:
 * calls that overlap on the GPU race, so serialise them.  d_coeffs must be
 * 8-byte aligned (BPC_ERR_ARG otherwise). */
int bpc_encode_compact_noalloc(const int *d_coeffs, int X, int Y, const int *d_lut, int lut_n, int passes, int levels,
                               int cb_size, int *d_compact, long long *d_offsets, int *d_status, void *stream);

/* ---------------------------------------------------------------------------
 * Request server (no counterpart in the reference, whose CUDA_BPC codes one
 * image per synchronous call).  Encode and decode requests of mixed size,
 * pass count, DWT depth and codeblock size are admitted in arrival order
 * against a device-memory budget and run concurrently, one launch per request
 * on up to max_in_flight streams, from a worker thread.
 *
 * Memory: bpc_server_create reserves budget_bytes of device memory once; each
 * request's output (encode: the X*Y-int slot stream; decode: X*Y coefficients)
 * is carved from it when the request is admitted and given back by
 * bpc_server_release.  Nothing is allocated while requests are served.  Inputs
 * (coefficients or slot streams) and LUTs are the caller's device buffers and
 * must stay valid until the request completes.  Unlike the rest of this
 * header, the bpc_server_* calls may be made from several host threads.
 * Requests run on streams of three priority classes by size (small first);
 * set CUDA_DEVICE_MAX_CONNECTIONS=32 in the environment before CUDA
 * initialises so that these streams do not share hardware queues (with the
 * default 8, a small request can wait behind a large one in the same queue).
 * ------------------------------------------------------------------------- */
int bpc_server_create(long long budget_bytes, int max_in_flight, void **server);
/* Register a device LUT (from bpc_load_luts) for a pass count and DWT depth;
 * *lut_id names it in bpc_server_submit.  The server does not own it. */
int bpc_server_register_lut(void *server, const int *d_lut, int lut_n, int passes, int levels, int *lut_id);
/* Queue a request; returns its ticket (>= 0) or a negative BPC_ERR_*
 * (BPC_ERR_TOO_LARGE when its output exceeds the whole budget). */
long long bpc_server_submit(void *server, int direction, const int *d_in, int X, int Y, int lut_id, int cb_size);
/* Withdraw a request that has not been admitted yet; it is then reported by
 * bpc_server_poll with status BPC_ERR_CANCELLED and no output. */
int bpc_server_cancel(void *server, long long ticket);
/* Take up to max finished requests (waiting up to wait_us for the first):
 * ticket, output (device; NULL if the request failed before running),
 * latency from submission to completion in microseconds, and status (0, the
 * OR of BPC_ST_* bits, or a negative BPC_ERR_*).  *n = number returned. */
int bpc_server_poll(void *server, int max, int wait_us, long long *tickets, int **outputs, double *latency_us,
                    int *status, int *n);
/* Give a finished request's output back to the budget. */
int bpc_server_release(void *server, const int *output);
int bpc_server_state(void *server, long long *queued, long long *in_flight, long long *bytes_used,
                     long long *completed);
/* Drops queued requests, waits for those on the GPU, frees the budget (every
 * output not yet released becomes invalid). */
int bpc_server_destroy(void *server);

/* ---------------------------------------------------------------------------
 * Per-codeblock stream files: the reference's load_CStream
 * (source/main_example.cu:51-68) over the file numbering of its load_Data
 * (:71-179).  File k is "<folder><k>.bin" (folder is a prefix, normally ending
 * in '/'): the cb_size*cb_size words of one codeblock's slot as 16-bit
 * big-endian values.  Files are numbered LL band first, then for level =
 * levels..1 the HL, LH and HH bands, each in raster order of codeblocks; file
 * k belongs to the slot of the codeblock at that position.  On reading, a byte
 * past the end of a file makes its word -1 (as fgetc's EOF does in the
 * reference); a missing file returns BPC_ERR_FILE.  The -1 fill of a slot is
 * written as 0xFFFF and reads back as 65535 (a decoder never reads it).
 * ------------------------------------------------------------------------- */
int bpc_load_cstreams(const char *folder, int *stream, int X, int Y, int levels, int cb_size);
int bpc_save_cstreams(const char *folder, const int *stream, int X, int Y, int levels, int cb_size);
/* Number of files the two calls above read or write for this geometry. */
int bpc_cstream_files(int X, int Y, int levels, int cb_size);

/* ---------------------------------------------------------------------------
 * LUT training (no counterpart in the reference, which ships trained tables
 * but no trainer).  A LUT entry is the probability, out of 128, that the
 * symbol coded with it is 0.  bpc_lut_stats adds to d_stats (device, 2 *
 * bpc_lut_entries(passes, levels, 15) unsigned 64-bit counters, zeroed by the
 * caller before the first image) the number of symbols the encoder codes with
 * each entry on the X x Y coefficients d_coeffs ([2k]) and how many of them
 * are 1 ([2k+1]), over planes 0..14; call it once per training image.
 * bpc_lut_write turns host counts into ref.txt, sig.txt, sign.txt (+ cp_sig.txt,
 * cp_sign.txt for 3 passes) in `folder` (a prefix, normally ending in '/'):
 * P = round(128 * zeros / symbols) clamped to 1..127, 64 where no symbol was
 * coded, each (level, subband) group listing planes up to one past its last
 * used plane, which is written as all 64 (the shipped tables' convention;
 * load_LUTs overwrites the last listed plane of a group with 64 after its
 * first entry), and the LL group listing all 15 planes so that load_LUTs
 * builds the 15-plane layout.  The files load with load_LUTs / bpc_load_luts.
 * ------------------------------------------------------------------------- */
int bpc_lut_stats(const int *d_coeffs, int X, int Y, int passes, int levels, int cb_size,
                  unsigned long long *d_stats, void *stream);
int bpc_lut_write(const char *folder, const unsigned long long *h_stats, int passes, int levels);

/* Reversible CDF 5/3 lifting DWT (JPEG 2000 integer filter) on the GPU, in
 * place on an X x Y int32 raster, `levels` levels, Mallat layout (LL top-left,
 * HL top-right, LH bottom-left, HH bottom-right) -- the input format of the
 * coder.  No counterpart in the reference, which takes pre-transformed data.
 * d_tmp: device scratch of X*Y ints.  X and Y must be multiples of 2^levels. */
int bpc_dwt53_forward(int *d_data, int X, int Y, int levels, int *d_tmp, void *stream);
int bpc_dwt53_inverse(int *d_data, int X, int Y, int levels, int *d_tmp, void *stream);

/* Number of ints of the loader array for a LUT folder's bitplane count. */
int bpc_lut_entries(int passes, int levels, int max_bitplane);

int bpc_version(void);

#ifdef __cplusplus
}
#endif

#endif /* BPC_PACO_H */
