/*
 * ampcor_b200: C ABI of the B200 (sm_100a) batched tile correlator.
 *
 * This is the drop-in boundary for the CUDA worker of ampcor.  Each entry point names the
 * reference interface it replaces (paths inside the isce-framework/ampcor source tree).
 * Every function returns AMPCOR_OK (0) or one of the AMPCOR_E_* codes and never throws; the
 * message of the last failure on a handle is available from ampcor_last_error().
 * All pointers are plain pointers; nothing here needs a C++ or PyTorch type.
 */
#ifndef AMPCOR_B200_H
#define AMPCOR_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* status codes (the reference raises std::bad_alloc / std::runtime_error / std::logic_error
   from its launchers, e.g. lib/libampcor_cuda/correlators/Sequential.icc:301-335) */
#define AMPCOR_OK 0
#define AMPCOR_E_ARG 1      /* invalid argument (null pointer, pair id out of range, ...) */
#define AMPCOR_E_SHAPE 2    /* tile geometry this build does not support */
#define AMPCOR_E_CUDA 3     /* CUDA runtime failure */
#define AMPCOR_E_NOMEM 4    /* host or device allocation failure */
#define AMPCOR_E_BOUNDS 5   /* a chip or window leaves its raster (the pair's offsets are NaN) */
#define AMPCOR_E_STATE 6    /* call out of order */

/* ampcor_params.flags */
#define AMPCOR_FLAG_REF_COMPAT 1u  /* assemble offsets with the reference formula, which
                                      subtracts the refine margin a second time
                                      (lib/libampcor_cuda/correlators/offsets.cu:124-125) */
#define AMPCOR_FLAG_PLAIN_FP32 2u  /* correlate with FP32 fused multiply-adds (the plain form)
                                      instead of FFTs (the spectral form) or bf16x3 split
                                      products on the tensor cores */
#define AMPCOR_FLAG_DERAMP 4u      /* remove each complex chip's and neighbourhood's linear phase
                                      ramp (lag-one autocorrelation phases along samples and
                                      lines) before the band-limited refinement; the reference's
                                      _deramp (Sequential.icc:1094-1098) is an empty stub, placed
                                      where a phase ramp could not change the amplitudes anyway */

typedef struct ampcor_handle ampcor_handle;

/*
 * Worker geometry.  Replaces the arguments of the reference worker constructor
 * Sequential(pairs, refLayout, tgtLayout, refineFactor, refineMargin, zoomFactor)
 * (lib/libampcor_cuda/correlators/Sequential.h:64-67) as parsed by the extension's
 * sequential(points, (refLines, refSamples), (tgtLines, tgtSamples), refineMargin,
 * refineFactor, zoomFactor) (ext/ampcor_cuda/sequential.cc:40-73).
 * Tiles are square (ref_lines == ref_samples, tgt_lines == tgt_samples), as the reference
 * assumes (Sequential.icc:55-60); the search margin is (tgt - ref) / 2.
 */
typedef struct {
    uint64_t pairs;          /* number of tile pairs of the arena API (capacity) */
    uint64_t ref_lines;      /* chip shape */
    uint64_t ref_samples;
    uint64_t tgt_lines;      /* search window shape */
    uint64_t tgt_samples;
    uint64_t refine_factor;  /* upsampling factor of the refinement (reference default 2) */
    uint64_t refine_margin;  /* refinement margin around the coarse peak (default 8) */
    uint64_t zoom_factor;    /* zoom factor of the refined correlation surface */
    int32_t device;          /* CUDA device ordinal */
    uint32_t flags;          /* AMPCOR_FLAG_* */
} ampcor_params;

/* per-pair diagnostics of the last run */
typedef struct {
    int32_t coarse_u, coarse_v;    /* coarse correlation maximum (placement row, column) */
    int32_t top, left;             /* nudged corner of the refinement neighbourhood */
    int32_t refined_u, refined_v;  /* refined correlation maximum */
    int32_t fine_p, fine_q;        /* maximum of the zoomed surface */
    float coarse_peak;             /* coarse correlation maximum value */
    float refined_peak;            /* refined correlation maximum value (peak correlation) */
    float zoom_peak;               /* zoomed surface maximum value */
    float reserved;
} ampcor_pair_diag;

/*
 * A batch of tile pairs cut from two complex64 rasters (row-major, lines x samples, the SLC
 * layout of lib/libampcor/dom/SLC.icc:123-126).  Replaces the host tile arena filled pair by
 * pair (pkg/ampcor/correlators/CUDA.py:50-54) with a gather on the device: pair p correlates the
 * chip whose upper-left pixel is (ulhc[4p], ulhc[4p+1]) in ref against the search window whose
 * upper-left pixel is (ulhc[4p+2], ulhc[4p+3]) in tgt (Plan.py:160-170 computes these corners).
 */
typedef struct {
    const void* ref;            /* complex64 reference raster */
    int64_t ref_lines, ref_samples;
    const void* tgt;            /* complex64 secondary raster */
    int64_t tgt_lines, tgt_samples;
    const int32_t* ulhc;        /* 4 int32 per pair */
    uint64_t pairs;
    float* offsets;             /* out: 2 floats per pair, (dy, dx) */
    ampcor_pair_diag* diag;     /* out, optional */
    float* coarse_surfaces;     /* out, optional: pairs x C^2 coarse correlation surfaces */
    float* refined_surfaces;    /* out, optional: pairs x Cf^2 refined correlation surfaces */
} ampcor_job;

/* Create a worker bound to params->device.  Replaces Sequential<raster_t>::Sequential
   (lib/libampcor_cuda/correlators/Sequential.icc:173-234) and the extension's
   sequential() (ext/ampcor_cuda/sequential.cc:40-73). */
int ampcor_create(const ampcor_params* params, ampcor_handle** handle);

/* Release the worker and all its memory.  Replaces the capsule destructor
   (ext/ampcor_cuda/sequential.cc:274-286) and Sequential::~Sequential (Sequential.icc:160-170). */
int ampcor_destroy(ampcor_handle* handle);

/* Copy the R x R complex64 chip of pair pid (row stride in pixels) into the worker's arena.
   Replaces Sequential::addReferenceTile (Sequential.icc:15-28) and the extension's
   addReference() (ext/ampcor_cuda/sequential.cc:85-143). */
int ampcor_add_reference(ampcor_handle* handle, uint64_t pid, const void* tile,
                         uint64_t row_stride);

/* Copy the W x W complex64 search window of pair pid.  Replaces Sequential::addTargetTile
   (Sequential.icc:31-44) and addTarget() (ext/ampcor_cuda/sequential.cc:155-213). */
int ampcor_add_target(ampcor_handle* handle, uint64_t pid, const void* tile,
                      uint64_t row_stride);

/* Correlate every pair of the arena and return the offset field: 2 floats per pair, (dy, dx) in
   pair order, owned by the worker and valid until the next adjust or destroy.  Replaces
   Sequential::adjust (Sequential.icc:47-141) and the extension's adjust()
   (ext/ampcor_cuda/sequential.cc:225-271). */
int ampcor_adjust(ampcor_handle* handle, const float** offsets);

/* Copy the per-pair diagnostics of the last ampcor_adjust into host memory (pairs entries).
   No reference counterpart (the reference keeps no per-pair record). */
int ampcor_diagnostics(ampcor_handle* handle, ampcor_pair_diag* diag);

/* Correlate a batch given device-resident rasters, corners and outputs; enqueued on stream
   (a cudaStream_t, NULL for the worker's own stream) without waiting.  Replaces the arena
   push and adjust (Sequential.icc:291-339, :47-141) with a device-side tile gather.  Pairs
   whose tiles leave a raster get NaN offsets and make the next ampcor_synchronize() return
   AMPCOR_E_BOUNDS. */
int ampcor_correlate(ampcor_handle* handle, const ampcor_job* job, void* stream);

/* Wait for the work enqueued on the worker's stream (or stream, when not NULL) and report
   any bounds failure of the batches since the last call. */
int ampcor_synchronize(ampcor_handle* handle, void* stream);

/* Same as ampcor_correlate but every pointer of job is host memory: the call uploads the
   rasters and corners, runs the batch and copies the offsets (and optional outputs) back before
   it returns.  This is the end-to-end path of pkg/ampcor/correlators/CUDA.py:22-61.  In the
   spectral form the rasters go up in bands of rows while the pairs whose tiles are already up
   are correlated (same offsets as one upload first); with page-locked host rasters the upload
   then hides behind the correlation, with pageable ones it does not. */
int ampcor_correlate_host(ampcor_handle* handle, const ampcor_job* job);

/* Placements per axis of the coarse (C = W - R + 1) and refined (Cf = 2 f m + 1) surfaces and
   the zoomed surface dimension (Z = z Cf), for sizing the optional outputs. */
int ampcor_surface_dims(const ampcor_handle* handle, int32_t* coarse, int32_t* refined,
                        int32_t* zoomed);

/* Switch per-stage timing on (enable != 0) or off.  While on, every batch records CUDA events
   around each kernel launch on the batch's stream.  No reference counterpart (the reference
   prints wall-clock stage times to a debug journal channel, e.g. tests/libampcor_cuda/
   correlate.cc). */
int ampcor_profile(ampcor_handle* handle, int enable);

/* Device time (milliseconds) spent in the coarse, refinement and fine kernels and the number of
   those kernel launches since profiling was switched on or last read; waits for the recorded
   events and resets the counters. */
int ampcor_stage_times(ampcor_handle* handle, double* coarse_ms, double* refine_ms,
                       double* fine_ms, uint64_t* launches);

/* Correlate a batch like ampcor_correlate(), but without allocating anything: for callers that
   cannot allocate device memory while they run, such as applications whose own memory pool
   already owns the whole GPU, or real-time and on-board processing chains that forbid
   allocation after start-up.  No reference counterpart.
   params gives the geometry and the device (params->pairs is ignored); every pointer of job is
   device memory on that device; the work runs on stream (a cudaStream_t, NULL for the legacy
   default stream) and every call waits for that stream to finish before it returns (it reads the
   bounds counter back to the host), so a stream that is being captured into a CUDA graph is
   refused with AMPCOR_E_ARG.  All intermediates live in one fixed device array of about 41 MiB;
   a call takes at most 16384 pairs (more returns AMPCOR_E_ARG).  The CUDA runtime creates the
   array when this library's device code is first loaded on a device (with lazy module loading,
   at the first call that needs it), so make one call with job->pairs == 0 at start-up, before
   the application's own pool takes the GPU: it loads the device code, looks up the array's
   address and launches nothing; from then on the device holds the array until the process
   exits.  All calls share the array: calls that overlap on the GPU (other processes, or
   streams the caller does not order) race and must be serialised by the caller; calls from
   threads of one process are serialised by a lock, and a failed call still waits for its stream
   before it releases the lock.  A failure message, if errbuf is not NULL, is written to errbuf
   (errlen bytes). */
int ampcor_correlate_noalloc(const ampcor_params* params, const ampcor_job* job, void* stream,
                             char* errbuf, size_t errlen);

/* Device time (ms) and launch count per kernel kind since profiling was switched on or last read:
   [0] coarse correlation, [1] refinement, [2] fine correlation, [3] coarse placement statistics,
   [4] fine placement statistics, [5] zoom ([3]-[4] run in the tensor-core form only, [5] in the
   tensor-core and spectral forms); resets the counters.  No reference counterpart. */
int ampcor_kernel_times(ampcor_handle* handle, double* ms, uint64_t* launches);

/* The worker's correlation form: 2 spectral (FFT correlation in shared memory), 1 tensor cores
   (bf16x3 split products), 0 plain FP32 direct sums; -1 for a NULL handle.  The spectral form is
   the default wherever the geometry allows it (windows of at most 160 samples, refined windows
   included), then the tensor-core form (at most 128 placements per axis);
   AMPCOR_FLAG_PLAIN_FP32 selects the plain form.  No reference counterpart. */
int ampcor_form(const ampcor_handle* handle);

/* Choose the correlation form (form: 2 spectral, 1 tensor cores, 0 plain FP32, -1 unchanged) and
   the number of pairs refined per chunk (chunk: 0 unchanged), as an autotuner does.  Waits for
   the worker's stream.  No reference counterpart. */
int ampcor_configure(ampcor_handle* handle, int form, uint64_t chunk);

/* Failure-detection test hook (no reference counterpart; the reference has no bounded waits).
   The next `batches` batches of the worker (tensor-core or spectral form) make the first wait of
   their tensor-core zoom, and of the staged spectral correlation kernels, on a barrier that
   nothing completes, bounded at about a millisecond: every wait of those kernels is bounded in
   time, and an expired wait stops the kernel cleanly and is reported.  The kernels issue no work
   after it and write no offsets for those batches (a staged coarse stage leaves its pairs
   refinement corners inside their windows), and the ampcor_synchronize() that ends each of them
   returns AMPCOR_E_CUDA with a time-out message; the worker stays usable.  0 switches it off. */
int ampcor_inject_timeout(ampcor_handle* handle, int batches);

/* The number of pairs refined per chunk. */
int ampcor_chunk(const ampcor_handle* handle, uint64_t* chunk);

/* Message of the last failure on handle (or of the last failed ampcor_create when handle is
   NULL). */
const char* ampcor_last_error(const ampcor_handle* handle);

/* Replace the extension's version() and copyright() (ext/ampcor_cuda/ampcor_cuda.cc:25-27). */
const char* ampcor_version(void);
const char* ampcor_copyright(void);

#ifdef __cplusplus
}
#endif

#endif /* AMPCOR_B200_H */
