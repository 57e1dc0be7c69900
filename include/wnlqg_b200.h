/*
 * wnlqg_b200.h - C ABI of the B200 k-mesh response engine.
 *
 * The engine evaluates the WannierNLQG k-mesh response hot path on one NVIDIA B200:
 * Fourier interpolation of H(R), (iR)^n H(R) and A(R) onto k-points, the per-k Hermitian
 * eigensolve, the sum-over-states integrands and the k-mesh reduction.
 *
 * Every array crossing this boundary is plain host (or, for *_device entry points, device)
 * memory described by pointers and sizes.  Complex numbers are two interleaved doubles
 * (re, im), exactly like Julia's ComplexF64.  Multi-dimensional arrays use the memory layout
 * of the reference's column-major Julia arrays, so a Julia `ccall` can pass its arrays
 * without copying:
 *   hamiltonian_r[nw, nw, NR]    element (i, j, R) at complex offset i + nw*(j + nw*R)
 *   position_r[nw, nw, 3, NR]    element (i, j, a, R) at i + nw*(j + nw*(a + 3*R))
 *   overlap_r[nw, nw, NR]        like hamiltonian_r
 *   r_vectors[3, NR] (int64)     element (a, R) at a + 3*R
 *   lattice[3, 3]                element (i, j) at i + 3*j; row i is lattice vector i (Angstrom)
 *
 * Errors: every entry point returns a wnlqg_status; the message of the last failure on the
 * calling thread is available through wnlqg_b200_last_error.  Handles are reentrant per
 * handle; calls on one handle must not overlap.
 */
#ifndef WNLQG_B200_H
#define WNLQG_B200_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define WNLQG_API __attribute__((visibility("default")))
#else
#define WNLQG_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

typedef enum wnlqg_status {
    WNLQG_OK = 0,
    WNLQG_ERR_INVALID_ARGUMENT = 1,   /* reference: ArgumentError */
    WNLQG_ERR_DIMENSION_MISMATCH = 2, /* reference: DimensionMismatch */
    WNLQG_ERR_NONFINITE = 3,          /* non-finite model data or results */
    WNLQG_ERR_CUDA = 4,               /* a CUDA runtime call failed */
    WNLQG_ERR_OUT_OF_MEMORY = 5,
    WNLQG_ERR_UNSUPPORTED = 6,        /* request outside what this build implements */
    WNLQG_ERR_DEVICE_TIMEOUT = 7      /* a bounded device-side wait gave up */
} wnlqg_status;

/* Response kinds (one per reference task family). */
typedef enum wnlqg_response_kind {
    WNLQG_SHIFT_CURRENT = 1,      /* sigma^{abc}(omega), ConventionalShiftCurrent.jl */
    WNLQG_INJECTION_CURRENT = 2,  /* eta^{abc}(omega), ConventionalInjectionCurrent.jl */
    WNLQG_BERRY_CURVATURE = 3,    /* occupied-sum Omega^{ab}, ConventionalQuantumGeometry.jl:188-215 */
    WNLQG_QUANTUM_METRIC = 4,     /* band-sum internal g^{ab}, ConventionalQuantumGeometry.jl:321-355 */
    WNLQG_INTRINSIC_AHC = 5,      /* sigma^{ab} Fermi sea over the mu axis, IntrinsicHallOccupations.jl */
    WNLQG_BERRY_DIPOLE = 6,       /* D^{abc} Fermi surface over the mu axis, BerryMultipoleMoments.jl */
    WNLQG_SECOND_HARMONIC = 7,    /* seven-term chi/sigma^{abc}(omega; 2 omega), SecondHarmonicKernels.jl */
    WNLQG_JERK_CURRENT = 8,       /* ordered jerk (abcd)(omega), ConventionalJerkCurrent.jl */
    WNLQG_LINEAR_TRANSPORT_BERRY = 9, /* Berry-curvature channel of the dc linear transport conductivity
                                        over the mu axis (any temperature), S m^2 per k-point before BZ
                                        weights and cell volume: LinearTransportKernels.jl:100-163 */
    WNLQG_BERRY_DIPOLE_SEA = 10   /* D^{abc} Fermi sea over the mu axis: sum_n f(E_n) d_c Omega_n^{ab}
                                     with the reference's default finite-difference geometry (central
                                     difference of the band curvature at k +- h e_c, h =
                                     finite_difference_step); BerryMultipoleGeometry.jl:67-161,
                                     QuantumGeometryDerivatives.jl:193-228, BerryMultipoleDC.jl:56-62 */
} wnlqg_response_kind;

typedef enum wnlqg_broadening {
    WNLQG_GAUSSIAN = 0,
    WNLQG_LORENTZIAN = 1
} wnlqg_broadening;

typedef enum wnlqg_precision {
    WNLQG_PRECISION_FP64 = 0,   /* plain FP64 throughout */
    WNLQG_PRECISION_MIXED = 1   /* FP32 bulk arithmetic, FP64 where accuracy needs it */
} wnlqg_precision;

#define WNLQG_MAX_RESPONSES 8
#define WNLQG_MAX_COMPONENTS 81

/* Model description (mirrors TightBindingModel, src/Core/Models.jl:11-75). */
typedef struct wnlqg_model_desc {
    int64_t num_orbitals;
    int64_t num_r_vectors;
    const double *lattice;         /* [3,3] */
    const int64_t *r_vectors;      /* [3,NR] */
    const int64_t *r_degeneracies; /* [NR] */
    const double *hamiltonian_r;   /* complex [nw,nw,NR], eV */
    const double *position_r;      /* complex [nw,nw,3,NR], Angstrom; may be NULL (zero) */
    const double *overlap_r;       /* complex [nw,nw,NR]; NULL for orthogonal models */
} wnlqg_model_desc;

/* One requested response and its Cartesian components (0-based axes). */
typedef struct wnlqg_response_request {
    int32_t kind;                                   /* wnlqg_response_kind */
    int32_t num_components;
    int32_t components[WNLQG_MAX_COMPONENTS][4];    /* (a,b,c,d); unused slots ignored */
} wnlqg_response_request;

/* Task description (the fields of EffectiveTaskConfig, src/Runtime/Config.jl:95-175, that the
 * hot path reads). */
typedef struct wnlqg_task_desc {
    int32_t num_responses;
    wnlqg_response_request responses[WNLQG_MAX_RESPONSES];
    double fermi_energy;               /* eV */
    double temperature;                /* K */
    int32_t broadening_type;           /* wnlqg_broadening */
    double broadening;                 /* eV */
    double transition_window_factor;
    double denominator_regularization; /* eV; 0 selects the bare inverse */
    double degeneracy_threshold;       /* eV */
    int64_t num_photon_energies;
    const double *photon_energies;     /* eV */
    int64_t num_fermi_energies;        /* mu axis for AHC / Berry dipole */
    const double *fermi_energies;      /* eV */
    int32_t precision;                 /* wnlqg_precision */
    double fermi_surface_broadening;   /* eV; Gaussian width of -f' at T = 0 (Berry dipole) */
    double shg_low_frequency_broadening;    /* eV; second harmonic low-frequency width (reference 0.025) */
    double shg_intermediate_regularization; /* eV; second harmonic eta; 0 selects denominator_regularization */
    int32_t shg_eta_correction;             /* second harmonic: 1 adds the finite-eta C numerator (reference true) */
    int32_t band_window_size;               /* shift/injection pairs: bands around mu, widened to complete
                                               degeneracy groups (select_band_window, CalculationUtils.jl:71-90,
                                               TransitionScreening.jl:201-233); -1 = all bands */
    /* Explicit interband selection (cfg.band_selection = (conduction, valence),
       validate_interband_band_selection, CalculationUtils.jl:501-522; gate in _fill_transition_screen!,
       TransitionScreening.jl:32-94): with use_band_selection = 1 a shift / injection pair (n, m) is kept
       only if bit n of valence_bands and bit m of conduction_bands are set (0-based band indices, bit i
       of word i / 32); both groups nonempty, disjoint and below num_orbitals; band_window_size must be -1. */
    int32_t use_band_selection;
    uint32_t valence_bands[4];
    uint32_t conduction_bands[4];
    /* Wannier-center convention (WannierCenterConventionTransforms.jl:1-130): 0 = Convention II
       (reference default), 1 = Convention I: centres tau = Re diag A(R = 0), derivative factors
       R + tau_j - tau_i, home-cell connection A - tau, and the similarity D(k) = diag(exp(2 pi i
       k.tau_frac)); orthogonal models only. */
    int32_t wannier_center_convention;
    /* Spectral gap tolerance in eV (EffectiveTaskConfig.spectral_gap_tolerance, Config.jl:104, reference
       default 1e-10).  With denominator_regularization = 0 the exact geometry of shift / injection
       current, Berry curvature, quantum metric and Berry dipole requires every pair of bands at a
       k-point to be split by more than this (geometry_isolated_spectrum_minimum_gap,
       OrthogonalBandDerivatives.jl:66-82, called at PositionMatrixElements.jl:447-452); the linear
       transport Berry channel groups levels closer than 32 eps into blocks and rejects distinct
       levels split by no more than this (spectral_subspace_blocks, SubspacePositionMatrixElements.jl:5-22).
       The Berry dipole always requires pairs split by more than degeneracy_threshold
       (BerryMultipoleGeometry.jl:81, BerryMultipoleDriver.jl:162).  A point that fails makes the call
       return WNLQG_ERR_INVALID_ARGUMENT with the reference's message. */
    double spectral_gap_tolerance;
    /* Interband rate gamma_inter in eV of WNLQG_LINEAR_TRANSPORT_BERRY (the reference's gamma_inter_ev,
       Config.jl:101; 0 = the clean limit). */
    double linear_transport_gamma_inter;
    /* Cartesian step h in 1/Angstrom of WNLQG_BERRY_DIPOLE_SEA (the reference's finite_difference_step,
       Config.jl:153, default 1e-4); the shifted points are k +- h e_c in fractional coordinates
       (finite_difference_step_matrix, Core/Coordinates.jl:33-44).  Their spectra must pass the same
       isolation check as the centre (degeneracy_threshold), reported on the centre's row. */
    double finite_difference_step;
    /* Geometry backend of WNLQG_BERRY_DIPOLE_SEA (the reference's derivative_backend, Config.jl:113):
       0 = finite differences (the default; finite_difference_step), 1 = analytic, the six-partition
       contraction of the band derivatives at the centre only (orthogonal_bcd_partition_matrices!,
       Responses/QuantumGeometry/OrthogonalGeometryDerivatives.jl:24-102, with the band derivatives of
       MatrixElements/Interpolated/OrthogonalBandDerivatives.jl:123-245). */
    int32_t derivative_backend;
} wnlqg_task_desc;

typedef struct wnlqg_model wnlqg_model;   /* device-resident model */
typedef struct wnlqg_plan wnlqg_plan;     /* compiled task: channels, tiles, workspaces */

/* Library version string. */
WNLQG_API const char *wnlqg_b200_version(void);

/* Message of the last error on the calling thread (always NUL-terminated; may be empty). */
WNLQG_API wnlqg_status wnlqg_b200_last_error(char *buffer, size_t capacity);

/* Number of visible CUDA devices (0 when no driver or device). */
WNLQG_API int32_t wnlqg_b200_device_count(void);

/* Copy a model to device `device`.  Replaces the model load of read_wannier_tb /
 * TightBindingModel (src/IO/WannierTB.jl:53-127, src/Core/Models.jl:11-75). */
WNLQG_API wnlqg_status wnlqg_b200_model_create(const wnlqg_model_desc *desc, int32_t device,
                                     wnlqg_model **out_model);
WNLQG_API wnlqg_status wnlqg_b200_model_destroy(wnlqg_model *model);

/* Compile a task for a model: Fourier channel plan and real-space tiles
 * (prepare_real_space!, HamiltonianMatrixElements.jl:92-198 and PositionMatrixElements.jl:8-84),
 * per-batch workspaces sized for `max_batch` k-points.
 * Replaces the setup half of _run_integral_bundle_owned! (Runtime/Execution/IntegralDriver.jl:92-560). */
WNLQG_API wnlqg_status wnlqg_b200_plan_create(wnlqg_model *model, const wnlqg_task_desc *task,
                                    int64_t max_batch, wnlqg_plan **out_plan);
WNLQG_API wnlqg_status wnlqg_b200_plan_destroy(wnlqg_plan *plan);

/* Number of complex values one k-point contributes (all responses concatenated).
 * Per response: shift/injection/jerk [num_photon_energies x num_components],
 * second harmonic [num_photon_energies x num_components x 7 terms x 2 quantities] (the reference's
 * raw per-k (frequency, component, term, quantity) array of SecondHarmonicDriver.jl:146-171),
 * curvature/metric [num_components], AHC/dipole [num_fermi_energies x num_components];
 * the energy axis is fastest. */
WNLQG_API int64_t wnlqg_b200_plan_value_count(const wnlqg_plan *plan);

/* Sum over the Gamma-centred mesh points k_begin <= idx < k_end of (1/Nk) * value(k), the
 * reference's lane tensor (consume_point!, IntegralDriver.jl:820-874, with the mesh of
 * CalculationUtils.jl:265-292, first axis fastest).  `out` (host) receives
 * plan_value_count complex values.  Replaces the per-worker k loop of
 * execute_prepared_tasks! (TaskSamplingScheduler.jl:151-217) for one lane. */
WNLQG_API wnlqg_status wnlqg_b200_eval_mesh(wnlqg_plan *plan, const int64_t mesh[3], int64_t k_begin,
                                  int64_t k_end, double *out);

/* Same as wnlqg_b200_eval_mesh with a device output pointer, on `stream` (a cudaStream_t, or
 * NULL for the legacy default stream).  Asynchronous: the caller synchronises the stream. */
WNLQG_API wnlqg_status wnlqg_b200_eval_mesh_device(wnlqg_plan *plan, const int64_t mesh[3],
                                         int64_t k_begin, int64_t k_end, double *out_device,
                                         void *stream);

/* Several plans (for example models of different orbital counts) in one call: plan i sums its
 * mesh meshes[3*i..3*i+2] over [k_begin[i], k_end[i]) into outs_device[i] (device, plan value
 * count complex values), exactly as wnlqg_b200_eval_mesh_device.  Every plan works on its own
 * stream after `stream` (NULL = legacy default stream) and joins back into it, so the models'
 * kernels overlap on the device.  Asynchronous; all plans must live on one device.  Batches the
 * per-worker task loop of execute_prepared_tasks! (TaskSamplingScheduler.jl:151-217) across
 * tasks. */
WNLQG_API wnlqg_status wnlqg_b200_eval_mesh_many(wnlqg_plan *const *plans, int32_t count, const int64_t *meshes,
                                       const int64_t *k_begin, const int64_t *k_end,
                                       double *const *outs_device, void *stream);

/* Per-point values at arbitrary fractional k-points: k[3*n] (host), out[n*value_count]
 * complex (host).  This is the ResponsePointEvaluator / ResponseNodeEvaluator contract
 * (Runtime/Execution/ResponsePointEvaluation.jl:8-64) batched over n points, used by the
 * adaptive integrator (ResponseIntegration.jl:100-198). */
WNLQG_API wnlqg_status wnlqg_b200_eval_points(wnlqg_plan *plan, const double *kpoints, int64_t n,
                                    double *out);

/* Weighted sum over arbitrary points: out = sum_i weights[i] * value(k_i), with k[3*n] and
 * weights[n] on the host.  This is the lane contract for a symmetry-reduced mesh
 * (representatives with multiplicities / Nk, consume_point!, IntegralDriver.jl:820-874) and for
 * a batch of adaptive nodes whose rule weights are known. */
WNLQG_API wnlqg_status wnlqg_b200_eval_points_weighted(wnlqg_plan *plan, const double *kpoints,
                                             const double *weights, int64_t n, double *out);

/* Same as wnlqg_b200_eval_points_weighted with DEVICE arrays (kpoints_device[3*n],
 * weights_device[n], out_device complex [value_count]) on `stream` (NULL = legacy default
 * stream); asynchronous, the caller synchronises.  For adaptive integrators whose nodes are
 * generated on the device (ResponseCubatureTree.jl:112-143 batch evaluation). */
WNLQG_API wnlqg_status wnlqg_b200_eval_points_weighted_device(wnlqg_plan *plan, const double *kpoints_device,
                                                    const double *weights_device, int64_t n,
                                                    double *out_device, void *stream);

/* Weighted sum over mesh indices: out = sum_i weights[i] * value(k(indices[i])) with k the
 * Gamma-centred mesh point of each index (first axis fastest).  Indices and weights are host
 * arrays.  This is the symmetry-reduced mesh contract (representatives and multiplicities/Nk,
 * numerical_response_symmetry_plan in IntegralDriver.jl:169-180, 820-874); runs of consecutive
 * indices use the staged mesh contraction. */
WNLQG_API wnlqg_status wnlqg_b200_eval_mesh_weighted(wnlqg_plan *plan, const int64_t mesh[3],
                                           const int64_t *indices, const double *weights, int64_t n,
                                           double *out);

/* Per-k band data for diagnostics and tests: energies [n*nw] (ascending) and the
 * canonicalised eigenvectors [n*nw*nw] complex, column-major per k
 * (compute_spectrum!, HamiltonianMatrixElements.jl:279-300 and :6-25). */
WNLQG_API wnlqg_status wnlqg_b200_eval_spectrum(wnlqg_plan *plan, const double *kpoints, int64_t n,
                                      double *energies, double *eigenvectors);

/* Allocation-free spectrum (no counterpart in the reference).  For callers that cannot let this
 * library allocate device memory (their memory belongs to another pool allocator under a fixed
 * budget).  Inputs and outputs are caller-owned DEVICE arrays on the current device:
 * hamiltonian_r complex [nw,nw,NR], r_vectors int64 [3,NR], r_degeneracies int64 [NR],
 * kpoints [3*n] fractional; energies [n*nw] ascending, eigenvectors complex [n*nw*nw]
 * (canonical phases, column-major per k).  Scratch is a fixed 8 MiB device array inside the
 * library, so n*(NR + nw^2)*16 bytes must stay below 8 MiB (larger n is rejected with
 * WNLQG_ERR_INVALID_ARGUMENT); nw <= 32.  The first call on a device looks up the scratch
 * address (cudaGetSymbolAddress); make that first call before any stream capture.  All calls
 * share the one scratch array: calls whose GPU work overlaps (other streams, other threads)
 * race on it.  Asynchronous on `stream` (NULL = legacy default stream).  The call itself
 * allocates nothing, but the 8 MiB array (with the library's device code) is reserved on each
 * device when the CUDA runtime loads this library's module there; under lazy module loading
 * (CUDA_MODULE_LOADING=LAZY, the CUDA 12 default) that happens inside the first call on the
 * device.  A caller with a fixed device budget should therefore make one warm-up call per device
 * at initialisation, before it sizes its pool and before any stream capture. */
WNLQG_API wnlqg_status wnlqg_b200_spectrum_noalloc(int64_t num_orbitals, int64_t num_r_vectors,
                                         const double *hamiltonian_r, const int64_t *r_vectors,
                                         const int64_t *r_degeneracies, const double *kpoints,
                                         int64_t n, double *energies, double *eigenvectors,
                                         void *stream);

/* Refinement-proposer MLP (no counterpart in the reference: it ranks adaptive cells for
 * subdivision and never supplies an integrand value).  8 input features -> 3 tanh layers of
 * 64 -> 1 output; FP32 master parameters, BF16 weight copies in the products, FP32 accumulation;
 * mean-squared-error loss; Adam.  Arrays are host arrays: x[n*8], targets/outputs[n],
 * params/grad[wnlqg_b200_mlp_param_count()]. */
typedef struct wnlqg_mlp wnlqg_mlp;
WNLQG_API int64_t wnlqg_b200_mlp_param_count(void);
WNLQG_API wnlqg_status wnlqg_b200_mlp_create(int32_t device, uint64_t seed, wnlqg_mlp **out_mlp);
WNLQG_API wnlqg_status wnlqg_b200_mlp_destroy(wnlqg_mlp *mlp);
WNLQG_API wnlqg_status wnlqg_b200_mlp_get_params(wnlqg_mlp *mlp, float *params);
WNLQG_API wnlqg_status wnlqg_b200_mlp_set_params(wnlqg_mlp *mlp, const float *params);
WNLQG_API wnlqg_status wnlqg_b200_mlp_forward(wnlqg_mlp *mlp, const float *x, int64_t n, float *y);
WNLQG_API wnlqg_status wnlqg_b200_mlp_loss_grad(wnlqg_mlp *mlp, const float *x, const float *target, int64_t n,
                                      float *loss, float *grad);
WNLQG_API wnlqg_status wnlqg_b200_mlp_train(wnlqg_mlp *mlp, const float *x, const float *target, int64_t n,
                                  int32_t steps, float learning_rate, float *final_loss);

/* Device time in milliseconds of the last eval_mesh* call's dominant kernel and of the
 * whole call (CUDA events on the plan's stream). */
WNLQG_API wnlqg_status wnlqg_b200_plan_last_timing(const wnlqg_plan *plan, double *fourier_ms,
                                         double *eigen_ms, double *response_ms,
                                         double *total_ms);

/* Number of kernel launches issued by the last eval_mesh* call. */
WNLQG_API int64_t wnlqg_b200_plan_last_launch_count(const wnlqg_plan *plan);

/* Device-side errors of the asynchronous entry points (*_device, eval_mesh_many): call after
 * synchronising the stream they ran on.  Reports, and clears, a bounded device wait that gave up
 * (WNLQG_ERR_DEVICE_TIMEOUT) and a k-point whose spectrum fails the task's isolation contract
 * (WNLQG_ERR_INVALID_ARGUMENT, the reference's GEOMETRY_SINGLE_BAND_SPECTRUM_NOT_ISOLATED /
 * SPECTRAL_CROSS_BLOCK_GAP_UNRESOLVED message; see spectral_gap_tolerance).  The synchronous entry
 * points run the same checks themselves. */
WNLQG_API wnlqg_status wnlqg_b200_plan_status(wnlqg_plan *plan);

/* ---- CUDA graphs (no reference counterpart: the reference's worker loop calls its evaluator
 * point by point; here one captured graph replaces a whole call) ------------------------------
 * A graph holds the complete Fourier -> eigensolve -> response -> reduce chain of one call with
 * its arguments fixed: wnlqg_b200_eval_mesh_many's work for several plans (models of different
 * orbital counts on their own streams, forked from and joined to the launch stream), or
 * wnlqg_b200_eval_points_weighted_device's work for one plan on fixed device buffers (the caller
 * rewrites the k-points and weights between launches; cells of an uneven adaptive refinement are
 * padded to the captured count with weight-0 points).  Capture runs the call once directly, then
 * records it.  While a graph exists its plans cannot be destroyed or autotuned, and buffers a
 * later direct call outgrows are retired, not freed.  Launches are asynchronous on `stream`;
 * after synchronising, wnlqg_b200_graph_status reports a bounded device wait that gave up. */
typedef struct wnlqg_graph wnlqg_graph;
WNLQG_API wnlqg_status wnlqg_b200_graph_capture_mesh_many(wnlqg_plan *const *plans, int32_t count,
                                                const int64_t *meshes, const int64_t *k_begin,
                                                const int64_t *k_end, double *const *outs_device,
                                                wnlqg_graph **out_graph);
WNLQG_API wnlqg_status wnlqg_b200_graph_capture_points_weighted(wnlqg_plan *plan, const double *kpoints_device,
                                                      const double *weights_device, int64_t n,
                                                      double *out_device, wnlqg_graph **out_graph);
WNLQG_API wnlqg_status wnlqg_b200_graph_launch(wnlqg_graph *graph, void *stream);
WNLQG_API wnlqg_status wnlqg_b200_graph_status(wnlqg_graph *graph);
/* Kernels one launch of the graph runs. */
WNLQG_API int64_t wnlqg_b200_graph_kernel_count(const wnlqg_graph *graph);
WNLQG_API wnlqg_status wnlqg_b200_graph_destroy(wnlqg_graph *graph);

/* ---- Autotuner (no reference counterpart) -------------------------------------------------
 * Measures, on the mesh block [k_begin, k_end) of `mesh`, every eigensolver team size (32, 64 and
 * 128 threads per matrix; orthogonal models up to 32 orbitals), the FP32 eigensolver stage's
 * start (warm from the previous point along mesh runs and ordered batches, or cold from the
 * identity; orthogonal models on the team or CTA mixed-precision stages), every contraction
 * tile (1, 2 and 4 photon energies per thread; frequency-resolved responses), the FP64
 * response CTA width (256 or 512 threads; orthogonal models whose per-point working set fits
 * shared memory) and the grids of the second-harmonic kernels whose working sets live in global
 * memory (metric inputs: 1, 2, 4 CTAs per SM; second harmonic: the L2-resident grid, 1, 2 CTAs
 * per SM), and likewise the grids of response passes and eigensolver stages whose per-CTA working
 * sets live in global memory (large orbital counts), keeps the fastest of each in
 * the plan and remembers it for the process (key: device, orbitals, precision, geometry, photon
 * energies, value count), so later plans with the same key take it without measuring.  Every
 * candidate is a configuration the library runs anyway; the tile choice leaves results bitwise
 * unchanged, while the grid choices decide how points are split among CTAs, and so the order of
 * the partial sums: on the FP64 path they may change results in the last bits; on the mixed path
 * they also change which neighbour each point's FP32 eigensolve warm-starts from, so results
 * change within the mixed path's accuracy (about 1e-6 relative).  Times are CUDA-event milliseconds of the second of two runs; -1 = not a
 * candidate; 0 in a choice = not tunable for this plan. */
typedef struct wnlqg_autotune_report {
    int32_t eigh_team;             /* chosen threads per matrix (32, 64, 128), 0 = fixed variant */
    int32_t energies_per_thread;   /* chosen contraction tile (1, 2, 4), 0 = no energy axis */
    double eigh_ms[3];             /* eigensolve time with 32, 64, 128 threads per matrix */
    double response_ms[3];         /* response time with 1, 2, 4 energies per thread */
    int32_t from_cache;            /* 1 when the choice came from the process cache */
    int32_t warm_start;            /* chosen FP32 start: 1 warm, 0 cold, -1 = not tunable */
    double start_ms[2];            /* eigensolve time with a cold and a warm start */
    int32_t response_threads;      /* chosen FP64 response CTA width (256, 512), -1 = not tunable */
    double width_ms[2];            /* response time with 256 and 512 threads per CTA */
    int32_t metric_shg_grid;       /* chosen CTAs of the metric SHG input kernel, -1 = none */
    double metric_shg_grid_ms[3];  /* response time with 1, 2 and 4 CTAs per SM */
    int32_t shg_grid;              /* chosen CTAs of the SHG kernel's global working-set variant, -1 = none */
    double shg_grid_ms[3];         /* response time with the L2-resident grid, 1 and 2 CTAs per SM */
    int32_t response_grid;         /* chosen grid of response passes with global working sets
                                      (0 = each pass's L2-resident grid), -1 = none */
    double response_grid_ms[3];    /* response time with the L2-resident grids, 1 and 2 CTAs per SM */
    int32_t eigh_grid;             /* chosen grid of eigensolver stages with global working sets, -1 = none */
    double eigh_grid_ms[3];        /* eigensolve time with the L2-resident grid, 1 and 2 CTAs per SM */
} wnlqg_autotune_report;
WNLQG_API wnlqg_status wnlqg_b200_plan_autotune(wnlqg_plan *plan, const int64_t mesh[3], int64_t k_begin,
                                      int64_t k_end, wnlqg_autotune_report *report);

/* ---- Measured arithmetic peaks (no reference counterpart: the roofline denominators of the
 * engine's SM-bound stages) ---------------------------------------------------------------------
 * Dense throughput of the device in TFLOP/s, each from one timed launch of independent dependency
 * chains on every SM (about 20 ms each): FP64 tensor-core mma.sync.m8n8k4 (DMMA, the engine's FP64
 * products), FP64 FMA and FP32 FMA on the CUDA cores.  A pure compute probe: no memory traffic,
 * no waits. */
WNLQG_API wnlqg_status wnlqg_b200_measure_peaks(int32_t device, double *fp64_dmma_tflops, double *fp64_fma_tflops,
                                                double *fp32_fma_tflops);

#ifdef __cplusplus
}
#endif

#endif /* WNLQG_B200_H */
