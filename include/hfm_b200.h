/* hfm_b200 — C ABI of the B200-native eikonal solve path.
 *
 * Drop-in boundary for the reference HamiltonFastMarching solve path. The reference exposes one
 * entry point, `void Run(IO&)` (Headers/DispatchAndRun.h:224-244), behind a key-value IO object
 * (JMM_CPPLibs/JMM_CPPLibs/Output/IO.h:77-118, BaseIO.h:16-43) that its front-ends fill and read:
 * the FileHFM executable (Interfaces/FileHFM/FileHFM.cpp:12-26) and the pybind11 class HFMIO
 * (Interfaces/PythonHFM/src/main.cpp:11-47). The functions below are what such a front-end binds:
 * an opaque `hfm_io` store with the same key semantics and a `hfm_run` that solves on the GPU.
 *
 * Conventions: plain pointers and sizes, no exceptions across the boundary. Every function
 * returns HFM_OK (0) or a positive HFM_ERR_* code; the message of the last failure on an object
 * is available from hfm_io_last_error(). Host arrays are copied in and out (the caller keeps its
 * buffers), exactly as PythonIO::PySetArray/PyGetArray do (PythonIO.hxx:7-35).
 * Distinct hfm_io objects may be used from distinct threads concurrently.
 */
#ifndef HFM_B200_H
#define HFM_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define HFM_OK 0
#define HFM_ERR_KEY 1           /* missing key, wrong field kind (string/scalar/array)            */
#define HFM_ERR_VALUE 2         /* invalid value: shape mismatch, non-SPD metric, bad ordering    */
#define HFM_ERR_UNSUPPORTED 3   /* a reference option this library does not implement            */
#define HFM_ERR_CUDA 4          /* CUDA runtime failure (message carries cudaGetErrorString)      */
#define HFM_ERR_NOT_CONVERGED 5 /* solver iteration cap reached, or a bounded device wait expired */
#define HFM_ERR_NOMEM 6         /* device or host allocation failure                              */
#define HFM_ERR_ARG 7           /* null pointer or buffer too small                               */

typedef struct hfm_io hfm_io;

/* Array orderings of the reference IO layer (IO.h:36): index of the ordering names
 * "RowMajor", "ColumnMajor", "YXZ_RowMajor", "YXZ_ColumnMajor". */
#define HFM_ORDER_ROW_MAJOR 0
#define HFM_ORDER_COLUMN_MAJOR 1
#define HFM_ORDER_YXZ_ROW_MAJOR 2
#define HFM_ORDER_YXZ_COLUMN_MAJOR 3

/* Replaces constructing an IO object (FileIO, PythonIO). `default_ordering` is the ordering used
 * when the "arrayOrdering" key is absent: RowMajor for files (IO.h:40), YXZ_RowMajor for Python
 * (PythonIO.h:20). */
hfm_io *hfm_io_create(int default_ordering);
void hfm_io_destroy(hfm_io *io);

/* Setters: HFMIO::SetScalar / SetString / SetArray (main.cpp:19-22). Arrays are float64, `shape`
 * lists `ndim` extents in the caller's storage order (component axis last). */
int hfm_io_set_scalar(hfm_io *io, const char *key, double value);
int hfm_io_set_string(hfm_io *io, const char *key, const char *value);
int hfm_io_set_array(hfm_io *io, const char *key, const double *data, int ndim, const int64_t *shape);
/* Zero-copy variant of hfm_io_set_array (an extension: the reference always copies): the store
 * reads `data` in place, so the caller keeps it alive and unmodified until the key is replaced or
 * erased, or the store destroyed. Used by request loops that hand large fields to a server. */
int hfm_io_set_array_view(hfm_io *io, const char *key, const double *data, int ndim, const int64_t *shape);

/* Getters: HFMIO::GetScalar / GetString / GetArray (main.cpp:17-21).
 * hfm_io_get_string copies at most `cap` bytes including the terminating NUL and stores the full
 * length (without NUL) in *len. hfm_io_get_array_info reports depth and extents (up to max_ndim);
 * hfm_io_get_array copies `count` doubles (must equal the product of the extents). */
int hfm_io_get_scalar(hfm_io *io, const char *key, double *value);
int hfm_io_get_string(hfm_io *io, const char *key, char *buf, size_t cap, size_t *len);
int hfm_io_get_array_info(hfm_io *io, const char *key, int *ndim, int64_t *shape, int max_ndim);
int hfm_io_get_array(hfm_io *io, const char *key, double *out, size_t count);
/* Zero-copy read of an array (an extension): *data points into the store, valid until the key is
 * replaced or erased or the store destroyed; *ndim and shape[:max_ndim] receive its extents. */
int hfm_io_get_array_ptr(hfm_io *io, const char *key, const double **data, int *ndim, int64_t *shape,
                         int max_ndim);

/* Field inspection: HFMIO::HasField / EraseField / GetComputedKeys (main.cpp:25-27,
 * BaseIO.hxx:38-47, PythonIO.hxx:37-48). has_field returns 1/0 (negative on a null argument). */
int hfm_io_has_field(hfm_io *io, const char *key);
int hfm_io_erase_field(hfm_io *io, const char *key);
int hfm_io_computed_keys(hfm_io *io, char *buf, size_t cap, size_t *len);

/* Replaces `void Run(IO&)` (DispatchAndRun.h:224-244) followed by IO::UsageReport
 * (main.cpp:14, BaseIO.hxx:64-104): dispatches at run time on the "model" key
 * (Riemann2, Riemann3, ReedsShepp2, ReedsSheppForward2, Dubins2, Elastica2, ReedsShepp3, TTI3,
 * Isotropic2/3, Diagonal2/3),
 * solves on the current CUDA device and writes the outputs (values, nAccepted, MaxStencilWidth,
 * costSensitivity_i, ...) into `io`.
 * If `expected_model` is non-NULL the call fails when "model" names another model, as the
 * single-model FileHFM_<Model> executables do (DispatchAndRun.h:227-233). */
int hfm_run(hfm_io *io, const char *expected_model);

/* Reverse first variation for the inspectSensitivity keys now in `io`, from the device state of
 * the last hfm_run on `io` that had the key retainState = 1 (an extension: the reference
 * differentiates inside Run). Writes costSensitivity_i and seedSensitivity_i as hfm_run does,
 * without solving again; HFM_ERR_ARG if no solve was retained. The retained device memory is
 * released with the store or by the next hfm_run. */
int hfm_run_sensitivity(hfm_io *io);

/* Runs `n` stores as one batch: each is read as by hfm_run, then the instances of one stencil family
 * and precision (and the same tileSweeps/maxRounds) are solved together — one global tile space
 * over all of them, one persistent solver launch — and each store receives its own outputs.
 * Stores with inspectSensitivity are solved on their own. `codes` (may be NULL) receives each
 * store's status; the return value is the first non-zero status, or HFM_OK. The values are those
 * hfm_run produces for each store alone (the fixed point of every instance is independent of its
 * batch neighbours); solver statistics (solverRounds, tileActivations, executedUpdates,
 * GPUSolveTime) are those of the whole batch. Extends the reference's one-instance Run(IO&). */
int hfm_run_batch(hfm_io *const *ios, int n, const char *expected_model, int *codes);

/* ---------------------------------------------------------------------------------------------
 * Serving (an extension: the reference answers one Run(IO&) at a time). A server owns one
 * scheduler thread and a resident persistent solver per model family (Riemann2, Riemann3,
 * ReedsShepp2, per precision). A plain solve (arrival times only) is admitted, in arrival order,
 * while its estimated device footprint fits in the memory budget and fewer than max_batch
 * instances are resident: its stencils are built in the family's device arena and its tiles join
 * the running solver at its next slice; the solver releases each instance as soon as its own
 * tiles have converged (continuous batching: no request waits for a larger one, and requests that
 * arrive while others are on the GPU join them). Other requests (other models, geodesics,
 * sensitivities, variations, stopping criteria, activeNeighs or stencil exports) run through
 * hfm_run between slices. max_batch = 1 runs every request through hfm_run, one at a time.
 * `lanes` is not used. Each request's outputs are written into its own store, exactly as hfm_run
 * would; the store must stay alive and untouched until the request is released.
 */
typedef struct hfm_server hfm_server;
typedef struct {
    int device;              /* CUDA device ordinal                                           */
    int lanes;               /* unused (kept for the layout of this structure)                 */
    int max_batch;           /* resident instances at most (default 64, at most 256; 1: plain)  */
    double hbm_budget_bytes; /* admission budget; <= 0: 80% of the free device memory          */
} hfm_server_config;
typedef struct {
    unsigned long long submitted, completed, batches, max_batch, queued, running_batches;
    double budget_bytes, bytes_in_use, peak_bytes;
} hfm_server_stats;

/* NULL on failure (no device, no memory). */
hfm_server *hfm_server_create(const hfm_server_config *cfg);
/* Queues `io` (filled as for hfm_run); HFM_ERR_NOMEM if it alone exceeds the budget. */
int hfm_server_submit(hfm_server *s, hfm_io *io, uint64_t *ticket);
/* Waits for a request (timeout_s < 0: no limit); *status receives its hfm_run status.
 * Returns HFM_ERR_NOT_CONVERGED if the timeout expired first. */
int hfm_server_wait(hfm_server *s, uint64_t ticket, double timeout_s, int *status);
/* Forgets a completed request; times (may be NULL) receives submit, start and completion times in
 * seconds since the server was created. */
int hfm_server_release(hfm_server *s, uint64_t ticket, double *times);
int hfm_server_get_stats(hfm_server *s, hfm_server_stats *stats);
/* Finishes the queued and running requests, then stops the scheduler. batches counts solver
 * slices, max_batch the most instances resident at once, running_batches those resident now. */
void hfm_server_destroy(hfm_server *s);

/* Message of the last failure on `io` ("" if none). Valid until the next call on `io`. */
const char *hfm_io_last_error(hfm_io *io);

/* Device-resident solve of a Riemannian instance (zero-copy path for serving and batching).
 * No reference counterpart as a function: it performs what Run(IO&) does for the Riemann2/Riemann3
 * models (Headers/Specializations/Riemannian.h:41-61 stencils, HamiltonFastMarching.hxx:59-112 solve)
 * with `metric`, `walls` and the output `values` already in device memory (RowMajor, component
 * axis last, packed xx,xy,yy[,xz,yz,zz]). Seeds are host arrays of RowMajor linear indices.
 * The solve runs on `stream` (cudaStream_t, NULL = legacy default stream); the call returns when
 * `values` is complete. On failure a message is copied into `err` (up to errcap bytes). */
typedef struct {
    int ndim;                 /* 2 or 3 */
    int64_t dims[3];
    double grid_scale[3];
    int dual;                 /* nonzero: `metric` is the dual metric */
    int precision;            /* 64 (reference-exact path) or 32 (fast path) */
    int sweeps_per_tile;      /* 0: default */
    const double *metric;     /* device pointer */
    const uint8_t *walls;     /* device pointer or NULL */
    int64_t nseeds;
    const int64_t *seed_index;
    const double *seed_value;
    double *values;           /* device pointer, receives FP64 arrival times (+inf unreached) */
    void *stream;
} hfm_riemann_device_args;

typedef struct {
    int64_t n_accepted;       /* reached cells (the reference's nAccepted) */
    int max_stencil_width;
    double stencil_ms, solve_ms;
    int64_t rounds, tile_activations, local_solves;
} hfm_solve_stats;

int hfm_solve_riemann_device(const hfm_riemann_device_args *args, hfm_solve_stats *stats, char *err,
                             size_t errcap);

/* Riemann2 FP64 solve that allocates nothing. No counterpart in the reference: it exists for
 * callers that cannot let a library allocate device memory (a host allocator that reserves the
 * whole device, a fixed memory budget, or a loop that must not be stalled by the device-wide
 * synchronisation of cudaMalloc/cudaFree). All intermediate arrays live in one fixed 9,453,824-byte
 * device buffer owned by the library, present on every GPU that loads it until the process exits;
 * the caller passes the metric (`nx*ny*3` doubles, RowMajor, packed xx,xy,yy) and receives the
 * arrival times (`nx*ny` doubles) in its own device memory. Limits: nx*ny <= 262144 cells and
 * 1..1024 seeds (RowMajor linear indices, host arrays); larger inputs fail with HFM_ERR_VALUE.
 * Repeated seed indices keep their first value. The first call on a device looks up the buffer's
 * device address; every call reads convergence words back and waits for its stream, so the entry
 * point cannot be called inside a stream capture. Calls share the buffer: concurrent or
 * overlapping calls on the GPU race and must be serialised by the caller. Results are within
 * 1e-10 (relative max-norm) of hfm_solve_riemann_device with precision 64. */
int hfm_solve_riemann2_static_scratch(int64_t nx, int64_t ny, double grid_scale, const double *metric,
                                      int dual, int64_t nseeds, const int64_t *seed_index,
                                      const double *seed_value, double *values, void *stream, char *err,
                                      size_t errcap);

/* Number of CUDA kernels this library has launched in the process (launch accounting). */
int hfm_kernel_launches(unsigned long long *count);

/* Library identification and device presence check (no GPU work). */
const char *hfm_version(void);
int hfm_device_count(int *count);

#ifdef __cplusplus
}
#endif
#endif /* HFM_B200_H */
