/*
 * dg_gpu.h — C ABI of the B200 (sm_100a) engine for the DG elastic-wave time loop.
 *
 * Replaces the five per-step functions the reference's driver loop calls
 * (DG_leap_Frog_OpenMP.c:418-437):
 *   Absorb_Boundary     OpenMP_Function.c:5-6, 25-46
 *   source_kernel       OpenMP_Function.c:8, 49-58
 *   LU_Velocity         OpenMP_Function.c:12-15, 75-185
 *   LU_Stress_Elastic   OpenMP_Function.c:17-20, 188-306
 *   Record              OpenMP_Function.c:10, 61-72
 * with one context that owns the device copies of the set-up arrays and advances any number of
 * steps per call.  The host keeps the reference's role: it reads meshes and operator files,
 * runs the set-up of fun_DG.c and hands the resulting arrays (exactly as fun_DG.c produces
 * them: element-major doubles, 1-based `long` index maps) to dg_gpu_init.
 *
 * Conventions: every function returns DG_OK (0) or a negative DG_ERR_* code and never exits
 * the process; a context is used from one host thread at a time and owns one CUDA stream;
 * calls return after the device work they launched has finished unless stated otherwise.
 */
#ifndef DG_GPU_H
#define DG_GPU_H

#ifdef __cplusplus
extern "C" {
#endif

#define DG_OK 0
#define DG_ERR_ARG -1          /* null pointer, bad size, bad enum */
#define DG_ERR_CUDA -2         /* a CUDA call failed (message via dg_gpu_last_error) */
#define DG_ERR_NOMEM -3        /* device or host allocation failed */
#define DG_ERR_MESH -4         /* index maps inconsistent (index out of range, maps not P2 faces) */
#define DG_ERR_NONFINITE -5    /* the watchdog found NaN/Inf in the velocity fields */
#define DG_ERR_STATE -6        /* stepping past the wavelet table, fetch of an unknown item */
#define DG_ERR_UNSUPPORTED -7  /* Np != 6, Nfp != 3, more meshes than supported */
#define DG_ERR_NODEVICE -8     /* no CUDA device, or not an sm_100 device */
#define DG_ERR_ORIENTATION -9  /* a triangle with non-positive Jacobian (compact paths need CCW) */
#define DG_ERR_TIMEOUT -10     /* a wait between blocks (wavefront step, grid barrier of a persistent batch) reached its limit */

/* arithmetic of the time loop */
#define DG_FP64_REF 0    /* the reference's per-element Dx/Dz/Q/A/B arrays, its operation order,
                            no FMA contraction: bit-identical to OpenMP_Function.c */
#define DG_FP64 1        /* geometric-factor form (Dr, Ds, rx..sz, LIFT): FP64 fields */
#define DG_FP32 2        /* FP32 fields and arithmetic, factors computed in FP64 and rounded */
#define DG_FP32_KAHAN 3  /* FP32 with a compensated (Kahan) update of every field */

/* items for dg_gpu_fetch / dg_gpu_load */
#define DG_VX 0
#define DG_VZ 1
#define DG_TXX 2
#define DG_TZZ 3
#define DG_TXZ 4
#define DG_TRACE_X 5   /* [steps_done][n_rec] like the reference's record_x[time*Channel + k] */
#define DG_TRACE_Z 6
#define DG_ENERGY 7    /* one double: 1/2 sum_e J_e (rho |v|^2 + sigma:C^-1 sigma) with the P2 mass matrix */

#define DG_MAX_MESHES 64

typedef struct dg_gpu_ctx dg_gpu_ctx;

/* One mesh with its medium, shots and receivers: the arrays of DG_leap_Frog_OpenMP.c:main
 * after set-up (fun_DG.c producers in brackets). */
typedef struct {
	long K;                    /* Tri: number of triangles */
	int Np, Nfp;               /* must be 6 and 3 (P2) */
	long n_points;             /* Point_Num */
	const double *Point;       /* [n_points][2]                                    (Mesh_Input) */
	const long *Triangle;      /* [K][3] 1-based vertex ids                        (Mesh_Input) */
	const double *Vr, *Vs;     /* [Np][Np] gradient Vandermonde (read from Vr.txt / Vs.txt) */
	const double *inverV;      /* [Np][Np] (inverV.txt) */
	const double *V;           /* [Np][Np] (V.txt); used for the energy mass matrix, may be NULL */
	const double *S;           /* [3][Np][Nfp] face lift (DG_leap_Frog_OpenMP.c:306-314) */
	const long *ibe;           /* [3][Nfp] 1-based face nodes                      (IBE) */
	const long *Neighbor;      /* [K][3] 1-based, boundary -> 1                    (Neighbor_Edge) */
	const long *Node_Neighbor; /* [K][3][Nfp] 1-based                              (NeighborNodes) */
	const long *Edge_flag;     /* [K][3] 1 interior face, 0 outer boundary         (Neighbor_Edge) */
	const double *A, *B;       /* [K][5]                                           (Elastic_A_B) */
	const double *Dx, *Dz;     /* [K][Np][Np]  DG_FP64_REF only, else may be NULL  (Dx_Dz) */
	const double *Q;           /* [K][3][5][2] DG_FP64_REF only, else may be NULL  (Central_flux) */
	const double *absorb_fun;  /* [K][Np]                                          (Absorbing_Fun) */
	int n_shots;               /* shots advanced together (the driver's m loop) */
	const long *source;        /* [n_shots][2] (triangle, node) 1-based            (Get_Source) */
	const double *fun;         /* [n_shots][Np] source vector (DG_leap_Frog_OpenMP.c:233-246) */
	int n_rec;                 /* receivers, shared by all shots */
	const long *receiver;      /* [n_rec][2] (triangle, node) 1-based, stride 2    (Get_Receiver) */
	double dt;                 /* Calculate_Time_Step */
	long n_steps;              /* length of wavelet[] = steps this mesh runs */
	const double *wavelet;     /* [n_steps] Ricker_Source(t, dt, t0) */
} dg_gpu_mesh;

typedef struct {
	int precision;       /* DG_FP64_REF / DG_FP64 / DG_FP32 / DG_FP32_KAHAN */
	int device;          /* CUDA device ordinal */
	int reorder;         /* 1: renumber elements along a Hilbert curve of centroids for locality */
	int block_threads;   /* threads per block, 0: automatic (or autotuned) */
	int graph_steps;     /* steps per captured CUDA graph (plus one of a quarter of them for shorter
	                        calls), 0: automatic (100), <0: no graphs */
	int autotune;        /* 1: time candidate block sizes (and, for a batch of meshes, the persistent or
	                        two-launch step; for the wavefront step its persistent form and lag) at init */
	int watchdog_every;  /* check the velocity fields for NaN/Inf every k steps (0: off) */
	const char *tune_cache; /* file that keeps autotune results between runs (NULL: none) */
	int variant;         /* FP32 kernels: 0 automatic, 1 one (element, shot) per thread,
	                        2 packed FP32x2 kernels (two elements or two shots per thread; element-major
	                        state for two shots per thread), 3 the same with plane-major state for 2-16 shots */
	int wavefront;       /* one launch per step that keeps the state in flight in L2 (single FP32 mesh
	                        of 1, 2, 4, ..., 128 shots): 0 automatic (on from 16 shots), 1 on, -1 off */
} dg_gpu_opts;

typedef struct {
	double ms_velocity;  /* device time of the last timed velocity half-steps (sum) */
	double ms_stress;    /* device time of the last timed stress half-steps (sum) */
	long launches;       /* kernels launched by the last dg_gpu_step/dg_gpu_step_timed */
	long steps_done;     /* steps taken so far (the `time` of the reference loop) */
	int block_threads;   /* block size in use */
	int graph_steps;     /* steps per graph in use */
	double bytes_per_step; /* algorithmic HBM bytes one step of all meshes moves */
	double dof_per_step;   /* 30 * sum over meshes of K * n_shots */
	int kernel_family;     /* 0 reference operators, 1 one (element, shot) per thread,
	                          2 two shots per thread (packed FP32x2), 3 two elements per thread (packed),
	                          4 FP32 batch of meshes, each block running its mesh's packed body,
	                          5 wavefront step (one launch per step, two shots per thread, one block per ticket),
	                          6 the same with resident blocks that loop over the tickets (FP32 default),
	                          7 two shots per thread on plane-major state (FP32, 2-14 shots),
	                          8 FP32 batch of meshes in one persistent cooperative launch for many steps,
	                            the bodies of 4 with a grid barrier between the halves (default for
	                            batches of at least 16 work blocks per resident block) */
} dg_gpu_stats;

void dg_gpu_default_opts(dg_gpu_opts *opts);

/* Copy the meshes to the device and prepare the kernels.  The host arrays may be freed
 * afterwards.  State starts at zero (the per-shot memset of DG_leap_Frog_OpenMP.c:412-416). */
int dg_gpu_init(dg_gpu_ctx **ctx, const dg_gpu_mesh *meshes, int n_meshes, const dg_gpu_opts *opts);

/* Advance every mesh by n steps (meshes whose n_steps are reached stay put).
 * Stepping past the longest wavelet table returns DG_ERR_STATE without doing anything. */
int dg_gpu_step(dg_gpu_ctx *ctx, long n);

/* The same steps, enqueued on the context stream without waiting for them (with the NaN
 * watchdog on, its checks still wait): the host is free until dg_gpu_synchronize, which waits
 * and reports a wait limit reached on the way (DG_ERR_TIMEOUT).  Every other call of the context
 * is ordered after the enqueued steps (fetches wait for them), except dg_gpu_fetch_traces of
 * steps an earlier step call completes and dg_gpu_set_wavelet of samples no enqueued step reads,
 * which run on a second stream while the later steps keep running. */
int dg_gpu_step_async(dg_gpu_ctx *ctx, long n);
int dg_gpu_synchronize(dg_gpu_ctx *ctx);

/* Same, timing each velocity and stress half-step with CUDA events on the context stream;
 * the sums land in dg_gpu_stats (ms_velocity, ms_stress). */
int dg_gpu_step_timed(dg_gpu_ctx *ctx, long n);

/* Advance n steps with a CUDA event before, between and after the two launches of every step,
 * all on the context stream and without host synchronisation until the end.  ms_vel / ms_str
 * (n floats each, may be NULL) receive each launch's device time (the wavefront step is one
 * launch: its time lands in ms_vel, ms_str holds about 0); ms_total the time from the
 * first event to the last.  With flush_l2 != 0 a buffer larger than L2 is written before every
 * step, outside the timed launches (ms_total then counts launches only). */
int dg_gpu_step_profiled(dg_gpu_ctx *ctx, long n, int flush_l2, float *ms_vel, float *ms_str, double *ms_total);

/* Receiver traces of steps [t0, t0+n) for every shot of one mesh:
 * dst_x / dst_z = double[n_shots][n][n_rec] (each shot like the reference's record_x window).
 * mesh = DG_ALL_MESHES: those blocks of every mesh one after the other, in mesh order, with one
 * synchronisation.  The call waits for the steps that wrote the window and returns with the
 * copies done; when a dg_gpu_step / dg_gpu_step_async call ended at or past step t0+n, it waits
 * for that call's steps only, so steps enqueued after it keep running meanwhile (a fetch of
 * chunk c overlaps the steps of chunk c+1). */
#define DG_ALL_MESHES (-1)
int dg_gpu_fetch_traces(dg_gpu_ctx *ctx, int mesh, long t0, long n, double *dst_x, double *dst_z);

/* Copy one item of one mesh/shot to host memory `dst`, in the reference's layout:
 * fields as double[K][Np] in the caller's element numbering, traces as double[steps][n_rec],
 * energy as one double.  For a field, shot = DG_ALL_SHOTS copies every shot of the mesh,
 * double[n_shots][K][Np], with one synchronisation. */
#define DG_ALL_SHOTS (-1)
int dg_gpu_fetch(dg_gpu_ctx *ctx, int what, int mesh, int shot, double *dst);

/* Overwrite one field of one mesh/shot from host memory (checkpoint restore); layout as fetch. */
int dg_gpu_load(dg_gpu_ctx *ctx, int what, int mesh, int shot, const double *src);

/* Zero every field and trace and rewind to step 0. */
int dg_gpu_reset(dg_gpu_ctx *ctx);

/* Replace wavelet samples [t0, t0+n) of one mesh with host values (the reference computes
 * w(t) on the host every step, DG_leap_Frog_OpenMP.c:421); mesh = DG_ALL_MESHES: w holds n
 * samples for each mesh, one after the other in mesh order.  Returns with w copied.  Steps
 * enqueued before the call that read these samples see the old ones; when none does (t0 at or
 * past the steps enqueued so far) the copy does not wait for the steps in flight. */
int dg_gpu_set_wavelet(dg_gpu_ctx *ctx, int mesh, long t0, long n, const double *w);

/* ---- one mesh split over several contexts (one per GPU): domain decomposition --------------
 * Replaces the reference's MPI driver (DG_leap_Frog_MPI.c:471-617), which keeps every array on
 * every rank and all-gathers the stresses and then the velocities of all partition-boundary
 * triangles twice per step (:486-558).  Here each context holds one part of the mesh: its own
 * triangles plus ghost copies of the neighbouring triangles of other parts (faces of a ghost
 * that lead out of the part are outer faces).  A step is
 *     dg_gpu_half_step(ctx, 0)   velocity half (sponge, source, LU_Velocity) on every element
 *     dg_gpu_halo_pack(ctx, m, 0, send) -> exchange -> dg_gpu_halo_unpack(ctx, m, 0, recv)
 *     dg_gpu_half_step(ctx, 1)   stress half (LU_Stress_Elastic, Record), ends the step
 *     dg_gpu_halo_pack(ctx, m, 1, send) -> exchange -> dg_gpu_halo_unpack(ctx, m, 1, recv)
 * The ghosts' own updates are wrong (some neighbours are missing) but are overwritten by the
 * exchange before any owned element reads them, so owned elements compute exactly what the whole
 * mesh computes.  Receivers and sources belong to the part that owns their triangle.  Needs the
 * two-launch step (opts.wavefront = -1). */

/* Velocity half (half = 0) or stress half (half = 1) of the next step, enqueued on the context
 * stream.  DG_ERR_STATE if the halves do not alternate; DG_ERR_UNSUPPORTED for a wavefront
 * context. */
int dg_gpu_half_step(dg_gpu_ctx *ctx, int half);

/* The same half step in two parts, so that the halo transfer overlaps computation: the boundary
 * part holds the elements with a ghost face neighbour (it must follow the unpack of the ghosts),
 * the interior part the other elements that are not ghosts (it needs no ghost value).  With the
 * halo lists set (they define the parts; one-mesh contexts only), an overlapped step is
 *     half_step_part(ctx, 0, INTERIOR)   while the previous step's stress halo is in transit
 *     unpack stresses; half_step_part(ctx, 0, BOUNDARY); pack velocities, start their transfer
 *     half_step_part(ctx, 1, INTERIOR)   while the velocity halo is in transit
 *     unpack velocities; half_step_part(ctx, 1, BOUNDARY); pack stresses, start their transfer
 * and owned elements compute exactly what dg_gpu_half_step computes, in any element numbering;
 * the overlap is largest when the boundary elements come first (opts.reorder = 0 and a mesh
 * numbered boundary, interior, ghosts).  Either part may run first; the half ends with the
 * second (which records, for the stress half).  DG_PART_ALL is dg_gpu_half_step.
 * DG_ERR_STATE if the halves do not alternate, a part runs twice or the other half's part is
 * missing, or no halo lists are set. */
#define DG_PART_ALL 0
#define DG_PART_BOUNDARY 1
#define DG_PART_INTERIOR 2
int dg_gpu_half_step_part(dg_gpu_ctx *ctx, int half, int part);

/* Elements (0-based, the mesh's own numbering) whose values this part sends, and the ghost
 * elements whose values it receives, each list in the order of the exchange buffers. */
int dg_gpu_halo_lists(dg_gpu_ctx *ctx, int mesh, long n_send, const long *send, long n_recv, const long *recv);

/* Copy the velocity (what = 0: Vx, Vz, 12 values per element and shot) or stress (what = 1:
 * Txx, Tzz, Txz, 18 values) planes of the send list into the device buffer `buf`, laid out
 * [element][plane][shot] in the context's arithmetic (8-byte doubles for the FP64 precisions,
 * 4-byte floats for the FP32 ones); returns once the buffer is filled. */
int dg_gpu_halo_pack(dg_gpu_ctx *ctx, int mesh, int what, void *buf);

/* The same copy, enqueued on the context stream without waiting for it: a caller that orders
 * its transfer after the context stream (a CUDA event recorded on dg_gpu_context_stream) and
 * the next half step and unpack after the transfer (the context stream waiting on an event of
 * the transfer's stream) steps a split mesh with no host synchronisation. */
int dg_gpu_halo_pack_async(dg_gpu_ctx *ctx, int mesh, int what, void *buf);

/* The context's CUDA stream (a cudaStream_t), on which every call of the context enqueues its
 * work: for ordering the caller's own work against it with events. */
void *dg_gpu_context_stream(dg_gpu_ctx *ctx);

/* Copy a device buffer of the same layout into the planes of the receive list (enqueued on the
 * context stream, ahead of the next half step). */
int dg_gpu_halo_unpack(dg_gpu_ctx *ctx, int mesh, int what, const void *buf);

/* Receives one velocity snapshot: step = steps done when it was taken, vx / vz = element-major
 * [K][Np] doubles of the mesh and shot asked for (the layout of dg_gpu_fetch), valid only
 * during the call. */
typedef void (*dg_gpu_snapshot_fn)(void *user, long step, const double *vx, const double *vz);

/* Advance n steps (a multiple of `every`) and hand Vx and Vz of (mesh, shot) to fn after every
 * `every` steps, while the device keeps stepping: snapshot j is copied on a second stream into
 * a pinned ring and fn(user, ...) runs on the calling thread while the device computes the
 * steps after it.  Replaces the reference's Save_Data of Vx/Vz every 100 steps
 * (DG_leap_Frog_OpenMP.c:433-444) without stalling the time loop; fn may write the files.
 * Returns after the last call of fn and the last step. */
int dg_gpu_step_snapshots(dg_gpu_ctx *ctx, long n, long every, int mesh, int shot, dg_gpu_snapshot_fn fn,
                          void *user);

/* Write a buffer larger than L2 on the context stream (timing hygiene between measurements). */
int dg_gpu_flush_l2(dg_gpu_ctx *ctx);

/* Test hook of the wavefront step (no counterpart in the reference): unit >= 0 makes the stress
 * update of that warp unit wait on a flag no warp ever publishes, so its wait reaches its limit
 * (about a second) and the next dg_gpu_step returns DG_ERR_TIMEOUT, the state of that step being
 * wrong; unit < 0 undoes it.  dg_gpu_reset then gives a context that steps as a fresh one.  On a
 * persistent batch of meshes (kernel family 8) unit >= 0 makes its grid barrier wait for one
 * block more than the grid holds, with a short limit (milliseconds), to the same effect.
 * DG_ERR_UNSUPPORTED when the context has neither. */
int dg_gpu_debug_stall_wave(dg_gpu_ctx *ctx, int unit);

/* Largest mesh dg_gpu_energy_noalloc accepts: its scratch holds one partial sum per 256 elements. */
#define DG_NOALLOC_MAX_ELEMENTS 4194304L

/* Energy of one wavefield, computed without allocating any device memory.
 * This entry point has no counterpart in the reference.  It serves callers that cannot call
 * cudaMalloc: for example an energy monitor called from inside another program's time loop,
 * where that program owns all device memory through its own pool and where a cudaMalloc or
 * cudaFree would synchronise the device and stall the running solver.
 * The caller passes every input and the output as device memory of `device`: the five fields
 * in the reference's layout (double[K][6] each), Jacobi[K] (Jacobian) and A[K][5] (Elastic_A_B:
 * 1/rho, 1/rho, lambda+2mu, lambda, mu); inverV is a host double[6][6] (inverV.txt); `out`
 * receives one double, the same quantity dg_gpu_fetch(..., DG_ENERGY, ...) returns.
 * Scratch: a file-scope static device array of DG_NOALLOC_MAX_ELEMENTS/256 doubles (128 KiB),
 * which every GPU that loads this library holds until the process exits.  K beyond
 * DG_NOALLOC_MAX_ELEMENTS is rejected with DG_ERR_ARG before anything runs.  The first call on a
 * device looks up the array's device address there (cudaGetSymbolAddress), with that device
 * current; a later call looks it up again only if the device's context has changed since (a
 * cudaDeviceReset by the host program).  Make the first call on each device, and the first one
 * after such a reset, before any stream capture.  Each call works on `device` and gives the
 * calling thread its previous current device back before it returns, on every path.  Launch
 * errors are read from the launches themselves: an error the host program left pending in the
 * CUDA runtime is neither returned nor cleared.  All calls share the array: calls that overlap
 * on the GPU (other streams, other host threads) race and give wrong results.  Each call
 * overwrites every partial it reads, so nothing has to start at zero.  `stream` is a
 * cudaStream_t (NULL: the default stream); the call returns after the result is in `out`. */
int dg_gpu_energy_noalloc(int device, long K, const double *Vx, const double *Vz, const double *Txx,
                          const double *Tzz, const double *Txz, const double *Jacobi, const double *A,
                          const double *inverV, double *out, void *stream);

int dg_gpu_stats_get(dg_gpu_ctx *ctx, dg_gpu_stats *out);
long dg_gpu_steps_done(dg_gpu_ctx *ctx);
int dg_gpu_free(dg_gpu_ctx *ctx);
const char *dg_gpu_strerror(int code);
/* Text of the last CUDA error seen by this thread ("" if none). */
const char *dg_gpu_last_error(void);

#ifdef __cplusplus
}
#endif
#endif
