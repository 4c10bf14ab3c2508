/*
 * twave.h - C ABI of the B200 (sm_100a) 2D staggered-grid SBP-SAT acoustic/elastic stepper.
 *
 * The reference (wsmoses/tpu-wave) has no plugin or FFI layer: its "API" is the C++ object
 * protocol that its two mains drive (cuda/src/cpp/main_host_FDM_2D.tpp:11-285 on the CPU,
 * cuda/src/cuda_main/nvcc_device_FDM_2D.cu:11-843 on the GPU). Each entry point below names
 * the reference member function or code block it replaces. Differences in convention:
 *   - every entry point returns a status (TW_OK = 0, negative on error) instead of printing and
 *     calling exit(0) (forward.cpp:37-98, cuda_container_run_time.cuh:57-62);
 *   - buffers are caller-owned host memory; `ld` arguments count elements;
 *   - one handle per host thread (handles are not thread-safe); handles are independent.
 *
 * Index conventions are the reference's: x is the slow data direction (rows), y the fast one;
 * the physical X axis is data y and physical Y is data x (namespace_forward.hpp:56-61).
 * Grids: TW_NN (Mx+1)x(My+1) "Sxy", TW_MN Mx x(My+1) "Vx" (velocity along data y),
 * TW_NM (Mx+1)x My "Vy" (velocity along data x), TW_MM Mx x My "SMM" = {sxx, syy}
 * (grid.hpp:146-188). Field readback uses exactly these (unpadded, row-major) sizes.
 */
#ifndef TWAVE_H
#define TWAVE_H

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#define TW_API __attribute__((visibility("default")))
#else
#define TW_API
#endif

/* ---- status codes --------------------------------------------------------------------- */
enum {
    TW_OK = 0,
    TW_ERR_INVALID = -1,        /* bad argument, size or enum */
    TW_ERR_CUDA = -2,           /* a CUDA runtime call failed (see tw_last_cuda_error) */
    TW_ERR_NOMEM = -3,          /* device or host allocation failed */
    TW_ERR_STATE = -4,          /* call out of order (e.g. stepping before the material is set) */
    TW_ERR_LOCATION = -5,       /* location is not a grid point (forward.cpp:38-39,48-49) */
    TW_ERR_OUTSIDE = -6,        /* location outside the grid (forward.cpp:91) */
    TW_ERR_WEAK_BOUNDARY = -7,  /* source on an SAT free-surface node row (forward.cpp:95-96) */
    TW_ERR_RECORD_FULL = -8,    /* more steps than the trace/energy records hold */
    TW_ERR_NONFINITE = -9,      /* a NaN/Inf appeared in a field (sticky, reported by tw_sync) */
    TW_ERR_UNSUPPORTED = -10,   /* combination not implemented (e.g. elastic with periodic x) */
    TW_ERR_MODEL_BOUNDS = -11,  /* interpolation stepped out of the model (grid_parameter.cpp:54-56) */
    TW_ERR_TOO_LARGE = -12,     /* model larger than the no-allocation scratch (TW_NOALLOC_MAX_MODEL_POINTS) */
    TW_ERR_IO = -13,            /* a file could not be opened, read or written, or is malformed */
    TW_ERR_TIMEOUT = -14        /* a wait inside a step kernel gave up (a staged copy did not arrive) */
};

/* ---- enums ------------------------------------------------------------------------------ */
enum tw_physics { TW_ELASTIC = 0, TW_ACOUSTIC = 1 };
/* x boundaries: SBP-SAT free surface (cuda/ tree), periodic (singlecore/ and mpi/ trees), or the
 * two x ends joined by the SBP-SAT interface penalty: the branch of secure_bdry for a boundary
 * type other than 'F' (grid_drvt.tpp:575-693, eta = +-1/2, every grid penalised toward the other
 * end's projection), which the reference's inputs never select (namespace_input.hpp:155-160).
 * y is periodic, as in the reference (grid_drvt.tpp:1-3), unless tw_grid_desc.sat_y is set. */
enum tw_bc { TW_BC_SAT_FREE = 0, TW_BC_PERIODIC = 1, TW_BC_SAT_INTERFACE = 2 };
/* storage type of the fields; FP64/FP32 compute in the storage type (namespace_type.cuh:16-22);
 * BF16/FP16 (elastic) store 16-bit fields, compute in FP32 and keep FP32 coefficients. The
 * reference's 16-bit mode (PRCSFLAG 16) also computes in 16 bits; this one rounds only what it
 * stores. */
enum tw_precision { TW_FP64 = 0, TW_FP32 = 1, TW_BF16 = 2, TW_FP16 = 3 };
/* time-update compensation, grid.hpp:550-566 / grid_update.tpp:1-127 ("N" = flops used for the
 * lost bits, "C" = separate array, "R" = the right-hand-side array holds them). Codes 1-6 need
 * FP64/FP32 storage. TW_CPST_SPLIT (no reference counterpart; BF16/FP16 only) is a compensated
 * (Kahan-style) two-term storage: each value is kept as hi + lo, lo = the rounding error of
 * hi, both 16-bit; the stencil, the energy and the receivers read the FP32 sum hi + lo, and the
 * update rounds the new FP32 value to hi and its remainder to lo. tw_read_field returns hi + lo,
 * tw_read_resid lo. */
enum tw_cpst { TW_CPST_00 = 0, TW_CPST_M3C = 1, TW_CPST_M3R = 2, TW_CPST_3C = 3,
               TW_CPST_3R = 4, TW_CPST_6C = 5, TW_CPST_6R = 6, TW_CPST_SPLIT = 7 };
enum tw_grid { TW_NN = 0, TW_MN = 1, TW_NM = 2, TW_MM = 3 };

typedef struct {
    int physics;            /* tw_physics */
    int bc_x;               /* tw_bc */
    int precision;          /* tw_precision */
    int cpst;               /* tw_cpst */
    long Mx, My;            /* cells along data x / y (ns_input::Mx_soln, My_soln) */
    int num_dx, den_dx;     /* dx = num/den (InputFile dxS, input_processing.cpp:63-72) */
    double dt;              /* ns_input::dt (main_host_FDM_2D.tpp:57) */
    double central_f;       /* Ricker central frequency (ns_input::central_f) */
    double time_delay;      /* Ricker delay (ns_input::time_delay) */
    double source_scaling;  /* divides the source increment (nvcc_device_FDM_2D.cu:557); 1 = none */
    int max_steps;          /* capacity of the trace and energy records */
    int energy;             /* 1: discrete energy every step (reference default, main_host_FDM_2D.tpp:34); 0: off */
    int device;             /* CUDA device ordinal (ns_input::device_number) */
    int coef_fp16;          /* 1: store the stepping coefficients in FP16 (elastic, FP32 arithmetic; no
                               reference counterpart): 10 B less per update; the medium is quantised to
                               FP16, and coefficients outside its normal range are TW_ERR_UNSUPPORTED.
                               2: store them as 16-bit fixed-point codes, each array on its own affine
                               map c = lo + step * code (lo its smallest value, step its range / 65535,
                               FP32 arithmetic): 16 significant bits across the array's range, 10 B less
                               per update (50 B with FP32 fields). Elastic, FP32 fields, TW_CPST_00, the
                               reference's boundaries, My >= 180 (the TMA-staged step reads the codes;
                               the other parts of the step read the decoded values). No reference
                               counterpart. tw_read_coefficients returns the values the step uses. */
    int sat_y;              /* 1: SBP-SAT free surfaces on the two y ends too (all four sides free with
                               bc_x TW_BC_SAT_FREE): closures and penalties along y with the x tables,
                               energy norm along y as along x; no reference run (its y is periodic).
                               0: periodic y (the reference). sat_y and TW_BC_SAT_INTERFACE need
                               FP64/FP32 storage; My >= 8 with sat_y */
} tw_grid_desc;

typedef struct {
    long rows[4], cols[4];  /* reference sizes of NN, MN, NM, MM */
    long pitch;             /* device row pitch in elements */
    int steps_done;
    int n_rcv;
    double bytes_per_update;       /* compulsory HBM bytes per cell-update of one step */
    double device_bytes;           /* device memory held by the handle */
    long row_off;                  /* a slab: global row of its local row 0 (0 otherwise) */
    long own_rows[2];              /* a slab: the global rows [own_rows[0], own_rows[1]) it owns */
    long Mx_glob;                  /* cells along x of the whole grid */
    int step_kind;                 /* how a step runs: 0 the per-point kernels (three or more launches),
                                      1 the one-launch fused step, 2 the TMA-staged step (two launches
                                      side by side), 3 the fused periodic acoustic step */
    int launches_per_step;         /* kernels one step launches */
} tw_info;

typedef struct tw_solver tw_solver;

/* Grid setup: Class_Grid::set_grid_parameters + set_forward_operators + set_grid_pointers for
 * the four grids (grid.hpp:146-481, called at main_host_FDM_2D.tpp:96-103) and the device
 * allocation of cuda_Class_Grid_initialize (grid.cuh:216-375). */
TW_API int tw_create(tw_solver **out, const tw_grid_desc *desc);
TW_API void tw_destroy(tw_solver *s);

/* Device memory of destroyed handles. A handle takes its buffers from a per-device memory pool
 * (stream-ordered) and tw_destroy returns them to it; the pool keeps them, so that creating the
 * next handle of a similar size maps no new memory (the reference allocates and frees per run,
 * grid.cuh:216-375 and cuda_container_run_time.cuh:268-275). This call gives the memory the
 * pool keeps on `device` back to the driver. No counterpart in the reference. */
TW_API int tw_release_cached_memory(int device);

/* Material from the reference's padded node model: Class_Grid::retrieve_forward_parameter,
 * define_parameters_energy, adjust_parameters_energy_periodic and make_density_reciprocal
 * (grid_parameter.cpp:7-160, grid_energy.cpp:8-177; main_host_FDM_2D.tpp:146-168).
 * rho/vp/vs: (Mx_prmt+2) x (My_prmt+2) doubles, row stride My_prmt+2 (inverse.cpp:79-90).
 * dxM = num_dxM/den_dxM is the model spacing. Acoustic handles use rho and vp only. */
TW_API int tw_set_material_model(tw_solver *s, const double *rho, const double *vp, const double *vs,
                          long Mx_prmt, long My_prmt, int num_dxM, int den_dxM);

/* Forward parameters given directly on one staggered grid (reference sizes, row stride ld):
 * NN idx 0 = mu; MN/NM idx 0 = rho (stored as 1/rho like make_density_reciprocal);
 * MM idx 0 = lambda (acoustic: kappa), idx 1 = 2mu. Replaces the material path for callers
 * that prepare coefficients themselves (the single-core tree sets them directly,
 * cpu_acoustic.cpp:178-180). */
TW_API int tw_set_material_grid(tw_solver *s, int grid, int idx, const double *coef, long ld);

/* The stepping coefficients the handle steps with, at reference sizes (row stride ld): NN idx 0
 * mu, MN / NM idx 0 1/rho, MM idx 0 lambda (acoustic: kappa), idx 1 2mu - the reference's
 * Vec_prmt after make_density_reciprocal (grid_parameter.cpp:131-160), rounded to the storage of
 * the handle (decoded from 16-bit codes with coef_fp16 = 2). */
TW_API int tw_read_coefficients(tw_solver *s, int grid, int idx, double *host, long ld);

/* Source: Class_Forward_Specs::process_src_locations (forward.cpp:10-100) with the location
 * given as rationals per data direction (struct_src_input, src_rcv.hpp:6-11). */
TW_API int tw_set_source_location(tw_solver *s, char type_x, char type_y, long num_x, long den_x,
                           long num_y, long den_y);
/* The same with grid indices. */
TW_API int tw_set_source(tw_solver *s, int grid, long ix, long iy);
TW_API int tw_clear_source(tw_solver *s);

/* Receivers: process_rcv_locations (forward.cpp:104-211). Appends in call order. */
TW_API int tw_add_receiver_location(tw_solver *s, char type_x, char type_y, long num_x, long den_x,
                             long num_y, long den_y);
TW_API int tw_add_receivers(tw_solver *s, int grid, const long *ix, const long *iy, int n);

/* Zero the fields, compensation arrays, records and the step counter (main_host_FDM_2D.tpp:225-235). */
TW_API int tw_reset(tw_solver *s);

/* Advance n steps: forward_simulation_periodic_y (forward_simulation.cpp:21-182) / the device
 * loop (nvcc_device_FDM_2D.cu:449-730). Asynchronous on the handle's stream. */
TW_API int tw_step(tw_solver *s, int n);
/* Wait for queued work; returns the first sticky error (TW_ERR_NONFINITE, TW_ERR_CUDA). */
TW_API int tw_sync(tw_solver *s);

/* Field readback in the reference layout (copy_field_pitched dev_to_hst, grid.cuh:463-469):
 * rows x cols of the grid, row stride ld >= cols, converted to double. field: 0, or 1 for syy on MM. */
TW_API int tw_read_field(tw_solver *s, int grid, int field, double *host, long ld);
/* Set a field from the host (reference layout). */
TW_API int tw_write_field(tw_solver *s, int grid, int field, const double *host, long ld);
/* Compensation arrays (Vec_rths for 'R' codes, Vec_cpst for 'C' codes), same layout. */
TW_API int tw_read_resid(tw_solver *s, int grid, int field, double *host, long ld);
TW_API int tw_write_resid(tw_solver *s, int grid, int field, const double *host, long ld);

/* Receiver traces: host[r][f][it] for r < n_rcv, f < 2, it < steps_done (Map_grid_RESULT_rcv,
 * forward.hpp:74-75; f = 1 is zero on single-field grids). */
TW_API int tw_read_receivers(tw_solver *s, double *host);
/* Energy records for it < steps_done (ns_input::Record_E_k/p0/p1). Elastic and acoustic-SAT:
 * E = E_k + (E_p0 + E_p1)/2 (forward.cpp:303-306). Acoustic periodic: E_k = E_Vx + E_Vy,
 * E_p0 = E_P of the previous step, E_p1 = E_P (cpu_acoustic.cpp:413-418). Any may be NULL. */
TW_API int tw_read_energy(tw_solver *s, double *E_k, double *E_p0, double *E_p1);

TW_API int tw_get_info(tw_solver *s, tw_info *info);
/* Advance n steps launching each kernel on its own, bracketed by CUDA events on the handle's
 * stream, and return the mean duration in ms of each phase: ms[0] velocity half-step,
 * ms[1] stress half-step, ms[2] energy reductions (all of one step), ms[3] receiver gather.
 * No counterpart in the reference, which times whole loops with steady_clock
 * (singlecore/src/main_cpp/cpu_acoustic.cpp:12-14,242-243). */
TW_API int tw_profile(tw_solver *s, int n, double *ms);
/* Rational location num/den of a node ('N') or cell-centre ('M') point -> grid index, as
 * process_src_locations / process_rcv_locations convert it (forward.cpp:31-51). Host only. */
TW_API int tw_location_to_index(char type, long num, long den, int num_dx, int den_dx, long *index);
/* The handle's cudaStream_t, for callers that order their own work after tw_step. */
TW_API int tw_get_stream(tw_solver *s, void **stream);
/* No counterpart in the reference: the material interpolation of tw_set_material_model without
 * any device allocation, for callers that cannot allocate device memory - a process whose GPU
 * memory is already reserved by another allocator (for example PyTorch's caching allocator) or
 * that fixes its memory budget at start-up, and that re-maps the medium repeatedly, as an
 * inversion loop does every iteration. tw_set_material_model allocates a temporary buffer per
 * call; this entry point uses a static device scratch of TW_NOALLOC_MAX_MODEL_POINTS doubles for
 * each of lambda, 2mu and mu on the padded model (12 MiB held by every GPU that loads the
 * library, until the process exits) and returns TW_ERR_TOO_LARGE for a larger padded model
 * (Mx_prmt+2)*(My_prmt+2). All pointers are caller-owned device memory: d_rho/d_vp/d_vs the padded
 * model (row stride My_prmt+2, d_vs zeros for acoustic media); outputs at the reference grid sizes,
 * compact: NN mu (Mx+1)x(My+1), MN rho Mx x(My+1), NM rho (Mx+1)x My, MM lambda and 2mu Mx x My -
 * the values tw_set_material_grid accepts. Runs on `stream` (a cudaStream_t, 0 for the legacy
 * default stream) and waits for it before returning. The first call on a device looks up the
 * scratch's device address (cudaGetSymbolAddress) with that device current; make that first call
 * before any stream capture. Every call shares the scratch, so calls that overlap on the GPU race. */
#define TW_NOALLOC_MAX_MODEL_POINTS (1L << 19)
TW_API int tw_material_map_noalloc(const double *d_rho, const double *d_vp, const double *d_vs, long Mx_prmt,
                                   long My_prmt, int num_dxM, int den_dxM, long Mx, long My, int num_dx,
                                   int den_dx, double *d_NN_mu, double *d_MN_rho, double *d_NM_rho,
                                   double *d_MM_lambda, double *d_MM_2mu, void *stream);

/* ---- slab decomposition ------------------------------------------------------------------
 * One elastic grid split along x (data rows) into slabs, each a handle of its own (its own GPU,
 * or all on one), a row decomposition as the reference's MPI tree exchanges halo strips
 * (mpi/src/cpp/namespaces.hpp:611-635), here four rows wide once per step, since a fused step
 * reaches four rows of the old state. tw_create_slab makes the handle of global rows
 * [row0, row1) of the grid `desc` describes (desc->Mx is the whole grid's): its arrays hold those
 * rows plus four halo rows at each edge that is not a free surface; the free-surface closures and
 * SAT terms apply only at the whole grid's top and bottom. Slabs need at least 16 rows, and at
 * least 16 rows from an inner cut to a free surface. Set-up takes the whole grid's terms: the model,
 * tw_set_material_grid arrays, source and receiver indices are global; a slab keeps the source
 * and the receivers in its own rows (the others record zeros, so traces and energies of all slabs
 * add up to the whole grid's). Field readback and writes are the slab's local arrays (halo rows
 * included; tw_get_info gives the offset and the owned rows). Step every slab, then exchange. */
TW_API int tw_create_slab(tw_solver **out, const tw_grid_desc *desc, long row0, long row1);
/* Refresh the halo rows of two vertically adjacent slabs (upper owns the rows just above lower's)
 * from each other's current state: device-to-device copies, any devices (peer or staged). Waits for
 * both handles' queued work first. A multi-GPU driver may instead move the same rows with NCCL,
 * through tw_slab_halo. */
TW_API int tw_slab_exchange(tw_solver *upper, tw_solver *lower);
/* The rows a slab sends or receives at one edge, for a caller's own transport (NCCL send/recv):
 * side 0 top, 1 bottom; recv 0: the owned rows the neighbour needs, 1: the halo rows to fill.
 * For field slot f (0 NN, 1 MN, 2 NM, 3 sxx, 4 syy; 5-9 their compensation arrays when present):
 * device pointer of the first row, row count, row length and row pitch in bytes, of the current
 * buffers (they alternate between steps). */
TW_API int tw_slab_halo(tw_solver *s, int side, int recv, int f, void **ptr, long *rows, long *row_bytes,
                        long *pitch_bytes);

/* The halo traffic of one edge as one contiguous device buffer, for a transport that moves
 * flat buffers (NCCL send/recv between ranks): tw_slab_pack copies the owned rows the neighbour
 * on `side` needs (every field, then every compensation array) into dst; tw_slab_unpack copies a
 * buffer packed by that neighbour into this slab's halo rows on `side`. *bytes (pack) is the
 * buffer size; call with dst NULL to learn it. Both run on the handle's stream. */
TW_API int tw_slab_pack(tw_solver *s, int side, void *dst, long *bytes);
TW_API int tw_slab_unpack(tw_solver *s, int side, const void *src);

/* Step the slabs of a whole grid together, `steps` steps, with the halo exchange fused into the
 * step kernel: while a slab's step writes its rows next to a cut, it also stores them straight
 * into the neighbour's halo rows of the same step's output buffers (peer stores over NVLink when
 * the neighbour is on another GPU of this process; peer access is enabled here, and
 * TW_ERR_UNSUPPORTED is returned where the GPUs cannot reach each other). Slab k's step waits on
 * its neighbours' previous step (CUDA events), so no step overwrites a halo row a neighbour still
 * reads. `slabs` lists every slab of the grid top to bottom (consecutive rows, the same step count
 * and set-up; FP32 / FP64 storage and coefficients, else TW_ERR_UNSUPPORTED); no tw_slab_exchange
 * is needed between or after the calls. Returns after queuing;
 * tw_sync each handle. No counterpart in the reference, whose MPI exchange is a separate
 * MPI_Sendrecv per halo strip (mpi/src/cpp/namespaces.hpp:611-635). */
TW_API int tw_slab_run(tw_solver *const *slabs, int n, int steps);

/* ---- adjoint gradient ---------------------------------------------------------------------
 * No counterpart in the reference (it has no adjoint). Full-waveform gradient of the misfit
 * J = 1/2 sum_{r,f,it} (trace[r][f][it] - obs[r][f][it])^2 by the discrete adjoint of the elastic
 * step (transposed SBP derivatives, closures and SAT penalties): a forward sweep of nt steps
 * from the handle's current state (steps_done must be 0) keeping a checkpoint every ckpt_every
 * steps, then a backward sweep that recomputes each segment from its checkpoint and steps the
 * adjoint through it. Elastic, compensation "00", FP64 or FP32 fields; gradients accumulate in
 * FP64. obs: [n_rcv][2][nt] like tw_read_receivers (entries of single-field receivers ignored).
 * Outputs (any may be NULL):
 *   misfit        J;
 *   g_grid[5]     dJ/d(material on each grid) at reference sizes: NN mu, MN rho, NM rho,
 *                 MM lambda, MM 2mu (the quantities tw_set_material_grid takes);
 *   g_rho/vp/vs   dJ/d(padded node model of tw_set_material_model), its layout ((Mx_prmt+2) x
 *                 (My_prmt+2)); TW_ERR_STATE when the material came from tw_set_material_grid;
 *   g_state[5]    dJ/d(initial fields NN, MN, NM, MM0, MM1) at reference sizes.
 * Afterwards the handle holds the state and records of tw_step(nt). Device memory for the call:
 * (nt/ckpt_every + ckpt_every + 2) states plus 15 field-sized arrays. */
TW_API int tw_adjoint_gradient(tw_solver *s, int nt, const double *obs, int ckpt_every, double *misfit,
                               double *const *g_grid, double *g_rho, double *g_vp, double *g_vs,
                               double *const *g_state);
/* The same gradient with binomial checkpointing (the revolve schedule family of Griewank and
 * Walther) in `slots` states: reversing n steps with c free slots advances a = min(n - 1,
 * C(c + t - 1, c)) steps into a slot, t the smallest number with C(c + t, c) >= n, and recurses on
 * both parts; the first advances are the forward sweep itself (traces and energies recorded once).
 * Device memory: slots + 5 states plus 15 field-sized arrays, for any nt; the forward steps taken
 * grow as memory shrinks (tw_revolve_plan). The gradient equals tw_adjoint_gradient's for any
 * slot count. No counterpart in the reference (it has no adjoint). */
TW_API int tw_adjoint_gradient_revolve(tw_solver *s, int nt, const double *obs, int slots, double *misfit,
                                       double *const *g_grid, double *g_rho, double *g_vp, double *g_vs,
                                       double *const *g_state);
/* The schedule of tw_adjoint_gradient_revolve alone (host only, no GPU): the forward steps it
 * takes for nt steps in `slots` states, and its number of actions; the schedule is replayed on
 * labels and checked (every adjoint step n meets the forward states n and n + 1). */
TW_API int tw_revolve_plan(int nt, int slots, long *forward_steps, int *n_actions);

/* Data misfit of the recorded traces against observed ones: calculate_data_misfit
 * (forward.cpp:414-445), sum over steps and fields of (trace - obs)^2 per receiver (no factor
 * 1/2: twice tw_adjoint_gradient's J), the difference taken in the storage precision for FP32
 * handles as the reference's FP32 build does. obs: [n_rcv][2][steps_done]; per_rcv may be NULL. */
TW_API int tw_data_misfit(tw_solver *s, const double *obs, double *total, double *per_rcv);

/* ---- batched shots ---------------------------------------------------------------------
 * No counterpart in the reference, which runs one shot per process. A batch advances many
 * acoustic handles (the shots: independent grids of any sizes) together: each half-step is ONE
 * launch over the tiles of all shots and one more launch records every shot's receivers, so
 * small shots no longer pay a launch per half-step each; G steps are replayed from a CUDA graph.
 * Each shot equals the same handle stepped alone with tw_step, bit for bit.
 * Requirements: acoustic handles on one device with the same precision (FP64/FP32),
 * compensation ('0', '3R', '6R') and x boundary, energy off, material set. The batch copies each
 * shot's set-up (source, receivers, buffers) at tw_batch_create: re-create it after changing a
 * shot's source or receivers. Shots stay usable on their own (readback, tw_step); tw_batch_step
 * orders itself after the shots' queued work and their later work after the batch. */
typedef struct tw_batch tw_batch;
TW_API int tw_batch_create(tw_batch **out, tw_solver *const *shots, int n);
TW_API void tw_batch_destroy(tw_batch *b);
/* Launch shape: blocks of tx x ty threads (tx*ty <= 256, a multiple of 32), rows_per_thread rows
 * per thread, `ctas` persistent CTAs walking the tile list (0: one CTA per tile). */
TW_API int tw_batch_set_shape(tw_batch *b, int tx, int ty, int rows_per_thread, int ctas);
TW_API int tw_batch_get_shape(tw_batch *b, int *shape4);
/* Autotuner: times `steps` batched steps for each candidate shape (tx in {32, 64, 128, 256},
 * 1/2/4 rows per thread, one CTA per tile or 4/8/16 persistent CTAs per SM), keeps the fastest
 * and returns its ms per step. It steps the shots, so it RESETS every shot afterwards
 * (tw_reset: fields, records and step counters zeroed); call it before setting initial fields. */
TW_API int tw_batch_tune(tw_batch *b, int steps, double *best_ms);
/* Advance every shot n steps (asynchronous); each shot's record must hold n more steps. */
TW_API int tw_batch_step(tw_batch *b, int n);
/* Wait for the batch; returns the first sticky error of any shot. */
TW_API int tw_batch_sync(tw_batch *b);

/* ---- the reference's files --------------------------------------------------------------
 * Readers and writers of the reference's own input and output files, so that workflows built
 * around its executables (InputFile.txt, SrcRcv.txt, model files, Signal / Energy / Snapshot
 * text outputs) can use this library unchanged. */
typedef struct {
    long Mx_prmt, My_prmt;      /* model_<X>_<Y>: model cells along data x, data y */
    long Mx, My;                /* grids_<X>_<Y>: simulation cells */
    int num_dxM, den_dxM;       /* dxM_<num>_<den>: model spacing */
    int num_dx, den_dx;         /* dxS_<num>_<den>: simulation spacing */
    char bdry[4];               /* bdry_<xL><xR><yL><yR>, upper case; zeros when absent */
    long Nt;
    double dt_max, cfl, dt;     /* MAXdt, CFL and dt = MAXdt * CFL (main_host_FDM_2D.tpp:57) */
    double central_f, time_delay;
    int device;
} tw_io_input;
/* InputFile.txt (input_processing.cpp:11-137); missing entries keep the reference's defaults. */
TW_API int tw_io_read_input(const char *path, tw_io_input *out);

typedef struct {
    long src_index;             /* the source's index (for a receiver: the source it belongs to) */
    long rcv_index;             /* the receiver's index; -1 for a source */
    char type_x, type_y;        /* 'N' or 'M' along data x, data y */
    long num_x, den_x, num_y, den_y;   /* location num/den along data x, data y */
} tw_io_point;
/* SrcRcv.txt (inverse.cpp:133-322): the Src and Rcv lines in file order. Writes at most cap
 * points; *n is the count in the file (cap 0 with pts NULL asks for it). A receiver listed
 * before its source is TW_ERR_IO, as the reference stops there. */
TW_API int tw_io_read_srcrcv(const char *path, tw_io_point *pts, int cap, int *n);
/* A model file (inverse.cpp:6-130): (Mx_prmt+1) x (My_prmt+1) native doubles, x outer, into the
 * padded (Mx_prmt+2) x (My_prmt+2) layout of tw_set_material_model (zeros in the padding). */
TW_API int tw_io_read_model(const char *path, long Mx_prmt, long My_prmt, double *padded);
/* Output files of the handle's records in the reference's text formats (forward.cpp:215-325,
 * nvcc_device_FDM_2D.cu:786-819), into `folder`:
 *   Signal_src_<s>_<src grid>_<iy>_<ix>_rcv_<r>_<rcv grid>_<iy>_<ix>.txt per receiver:
 *     "% 6d  " step, then "% 16.15e  " per field of the grid;
 *   Energy_src_<s>_<src grid>_<iy>_<ix>.txt (energy on): "%16.15e" of E_k + (E_p0 + E_p1) / 2;
 *   with snapshots != 0, Snapshot_<grid>_<name>_<field>.txt: the current field, row-major.
 * Grid strings list the data-y type first, as the reference writes them; values are multiplied
 * by source_scaling (the energy by its square). rcv_index: one index per receiver (NULL: 0, 1, ...). */
TW_API int tw_io_write_records(tw_solver *s, const char *folder, int src_index, const int *rcv_index, int snapshots);

TW_API const char *tw_strerror(int status);
TW_API const char *tw_last_cuda_error(void);

#ifdef __cplusplus
}
#endif
#endif
