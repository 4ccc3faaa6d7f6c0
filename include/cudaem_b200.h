/*
 * cudaem_b200.h -- C ABI of the B200 multislice engine.
 *
 * This is the drop-in boundary for the simulator surface of cudaEM.  Every
 * entry point below names the reference interface it replaces
 * (file:line inside the cudaEM source tree).  The reference exposes a C++
 * class `mulSimulator` whose methods take `multislice_params<float>` and
 * fill `output_Multi_Data<float>` (simulator.cu:8, :20, :31); both structs
 * live in headers that the reference does not ship (multislice_params.hpp,
 * output_multislice_data.hpp).  Their fields, as read by the reference
 * (multislice_params_dev.cuh:88-199, simulator.cu:13-46), are flattened into
 * the plain-old-data structs `ms_params` and `ms_output` below.
 *
 * Conventions
 *  - Grid: `nx` columns (fast index, x) by `ny` rows (y), row-major,
 *    sampling dx = lx/nx, dy = ly/ny (grid_dev.cuh:307-325).
 *  - All lengths in Angstrom, angles in rad, beam energy in kV, aberration
 *    coefficients in Angstrom.  Aperture and detector angles are converted
 *    to spatial frequency with g = sin(angle)/lambda.
 *  - Output scaling follows the reference exactly: forward FFTs are
 *    unnormalised, the Fresnel propagator carries 1/(nx*ny)
 *    (device_kernels.cuh:225), the exit wave stays in reciprocal space
 *    scaled by nx*ny (wave_function.cuh:71) and the probe is built by an
 *    unnormalised inverse FFT (incident_wave.cuh:37-39).
 *  - Every function returns an ms_status; on failure the context keeps a
 *    message readable with ms_last_error().  No function prints.
 *  - A context owns one CUDA stream and serves one host thread at a time.
 *    Calls block until their results are in the caller's buffers.
 */
#ifndef CUDAEM_B200_H
#define CUDAEM_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define MS_ABI_VERSION 2
#define MS_NR 128        /* radial spline nodes; c_nR in the reference (basic_functions_dev.cuh:51-65) */
#define MS_MAX_DET 8     /* annular detectors per simulation */
#define MS_MAX_COEF 6    /* linear / non-linear coefficients per element parameterisation */

typedef enum ms_status {
    MS_OK = 0,
    MS_ERR_INVALID_ARG = 1,   /* a parameter failed validation */
    MS_ERR_UNSUPPORTED = 2,   /* a mode or size this engine does not implement */
    MS_ERR_CUDA = 3,          /* a CUDA runtime call or kernel launch failed */
    MS_ERR_OUT_OF_MEMORY = 4, /* device allocation failed */
    MS_ERR_TIMEOUT = 5,       /* a bounded device-side wait ran out */
    MS_ERR_NO_DEVICE = 6,     /* no CUDA device, or the device index is out of range */
    MS_ERR_INTERNAL = 7
} ms_status;

/* eTEM_Sim_Type (single_simulator.cuh:439-450, scan_simulator.cuh:185-200) */
enum { MS_SIM_HRTEM = 1, MS_SIM_ED = 2, MS_SIM_CBED = 3, MS_SIM_STEM = 4 };
/* ePhonon_Model (multislice_params_dev.cuh:25) */
enum { MS_PHONON_STILL = 1, MS_PHONON_FROZEN = 3 };
/* eIncident_Wave_Type (incident_wave.cuh:29-46); MS_IW_PLANE_TILTED is the plane wave times the
 * beam-tilt factor exp(2 pi i g0.(r - L/2)) of Incident_Wave::apply_beam_tilt (incident_wave.cuh:72-78,
 * exp_r_factor_2d, device_kernels.cuh:519-533) with g0 = sin(theta)(cos phi, sin phi)/lambda */
enum { MS_IW_PLANE = 1, MS_IW_CONVERGENT = 2, MS_IW_PLANE_TILTED = 3 };
/* ePotential_Type (basic_functions_dev.cuh:187-214); MS_POT_MOLIERE is this engine's built-in table */
enum {
    MS_POT_DOYLE_0_4 = 1, MS_POT_PENG_0_4 = 2, MS_POT_PENG_0_12 = 3, MS_POT_KIRKLAND_0_12 = 4,
    MS_POT_WEICKENMEIER_0_12 = 5, MS_POT_LOBATO_0_12 = 6, MS_POT_MOLIERE = 7
};
/* eIllumination_Model (lens_modulation.cuh:34-54): coherent CTF, partially coherent CTF
 * (envelope, PCTF_TEM :91-110) or transmission cross-coefficient quadrature (TCC_TEM :130-176);
 * the last two apply to the HRTEM image */
enum { MS_ILLUM_COHERENT = 1, MS_ILLUM_PARTIAL = 2, MS_ILLUM_TCC = 3 };
/* eTemporal_Spatial_Incoh (multislice_params_dev.cuh:27) */
enum { MS_TSI_TEMPORAL_SPATIAL = 1, MS_TSI_TEMPORAL = 2, MS_TSI_SPATIAL = 3, MS_TSI_COHERENT = 4 };
/* data_record (multislice_params_dev.cuh:117): intensity or full complex wave */
enum { MS_RECORD_INTENSITY = 0, MS_RECORD_WAVE = 1 };
/* execution form of the STEM scan: batched probes on the whole specimen (tile scan,
 * run_STEM_tile_simu, scan_simulator.cuh:11-113); one probe per launch on the whole specimen
 * (the plain comparator); or the general scan (run_STEM_general_simu, scan_simulator.cuh:115-183):
 * per probe position the grid box is a window of lx x ly centred on the probe, the atoms of the
 * displaced specimen inside it +- 2 A are cropped and shifted into it, and a window without atoms
 * records the unscattered probe's detector intensity */
enum { MS_EXEC_BATCHED = 0, MS_EXEC_PLAIN = 1, MS_EXEC_GENERAL = 2 };
/* eMatch_Border for slicing (slice_generator.hpp:130-168) */
enum { MS_BORDER_MIN = 0, MS_BORDER_MAX = 1, MS_BORDER_MIDDLE = 2 };

/* Lens: the host lens of the reference, exported to Lens_Dev (lens_dev.cuh:74-131). */
typedef struct ms_lens {
    int m;                                   /* vortex momentum */
    double c10, c12, phi12, c21, phi21, c23, phi23;
    double c30, c32, phi32, c34, phi34;
    double c41, phi41, c43, phi43, c45, phi45;
    double c50, c52, phi52, c54, phi54, c56, phi56;
    double inner_aper_ang, outer_aper_ang;   /* aperture semi-angles, rad */
    /* partial coherence of the objective lens (lens_dev.cuh:27-34) */
    double dsf_sigma;                        /* standard deviation of the defocus spread, Angstrom */
    double ssf_beta;                         /* source divergence semi-angle, rad */
    int dsf_npoints;                         /* TCC: defocus quadrature points (Gauss-Hermite) */
    int ssf_npoints;                         /* TCC: source quadrature points per axis (Gauss-Hermite) */
} ms_lens;

/* One element's V(r) parameterisation: the cl/cnl tables of Element_Coeffs
 * (device_containers.cuh:208-285), in the functional form `form` (an
 * MS_POT_* value).  Elements not listed use the built-in Moliere table. */
typedef struct ms_element_coef {
    int Z;
    int form;
    double cl[MS_MAX_COEF];
    double cnl[MS_MAX_COEF];
} ms_element_coef;

/* Atom_Coord_Data<float>: structure of arrays, host memory, caller-owned. */
typedef struct ms_atoms {
    int64_t n;
    const int* Z;
    const float* x;
    const float* y;
    const float* z;
    const float* sigma;   /* per-axis r.m.s. thermal displacement, Angstrom */
    const float* occ;     /* occupancy */
} ms_atoms;

/* multislice_params<float>, restricted to the modes this engine implements. */
typedef struct ms_params {
    int simulation_type;          /* MS_SIM_* */
    int nx, ny;                   /* grid_2d.col, grid_2d.row: powers of two in [128, 2048] */
    double lx, ly;                /* box size, Angstrom */
    double dz;                    /* slice thickness, Angstrom */
    int bwl;                      /* band-width limit of the propagator (grid_dev.cuh:462-465) */
    double E0;                    /* beam energy, kV */
    double theta, phi;            /* beam tilt, rad */
    int potential_type;           /* MS_POT_* default form for elements without an explicit table */
    double pot_rmin, pot_rmax;    /* radial spline range (R_min, R_max), Angstrom; 0 selects 0.01 / 3.0 */
    int pot_wrap;                 /* 0: distance as the reference (no periodic images); 1: minimum image */
    const ms_element_coef* element_coefs;
    int n_element_coefs;
    int phonon_model;             /* MS_PHONON_STILL or MS_PHONON_FROZEN */
    int pn_nconf;                 /* number of frozen-phonon configurations */
    uint64_t pn_seed;             /* phonon seed */
    int pn_dim_x, pn_dim_y, pn_dim_z;  /* axes that vibrate (FP_Dim) */
    int slice_border;             /* MS_BORDER_*; -1 selects the reference rule (max for HRTEM, min otherwise) */
    int iw_type;                  /* MS_IW_*; -1 selects plane for HRTEM/ED and convergent for CBED/STEM */
    double iw_x, iw_y;            /* probe position in the specimen frame, Angstrom */
    ms_lens cond_lens;            /* condenser lens: the probe */
    ms_lens obj_lens;             /* objective lens: the HRTEM image */
    int illumination_model;       /* MS_ILLUM_* */
    int temporal_spatial_incoh;   /* MS_TSI_*: which spreads the partial-coherence models include */
    int data_record;              /* MS_RECORD_* */
    int scan_nx, scan_ny;         /* STEM scan size (columns, rows) */
    double scan_x0, scan_y0;      /* first probe position, Angstrom */
    double scan_dx, scan_dy;      /* scan step, Angstrom */
    int n_det;                    /* annular detectors */
    double det_inner[MS_MAX_DET]; /* inner semi-angle, rad */
    double det_outer[MS_MAX_DET]; /* outer semi-angle, rad */
    int thick_det;                /* detector whose annulus filters the thickness series (reference: 1) */
    int exec_mode;                /* MS_EXEC_* */
    int probe_batch;              /* probes per batch; 0 lets the autotuner choose */
    int ckpt_interval;            /* adjoint: store the wave every k slices (>= 1) */
    int enable_fine_slicing;      /* 1: per-slice integrated atom potentials (projected_potential.cuh:34-45, :94-133) */
    int gpu_num;                  /* must be 1: one GPU per context */
} ms_params;

/* output_Multi_Data<float>: caller-allocated buffers. */
typedef struct ms_output {
    float* image_intensity;       /* ny*nx: HRTEM image, ED / CBED pattern (fft-shifted) */
    float* image_real;            /* ny*nx: full wave, real part (data_record == MS_RECORD_WAVE) */
    float* image_imag;            /* ny*nx: full wave, imaginary part */
    float* stem_intensity;        /* n_det*scan_ny*scan_nx, laid out [det][row][col] */
    float* thickness_frames;      /* n_frames*ny*nx, laid out [slice][row][col] */
    int64_t thickness_capacity;   /* floats available in thickness_frames */
    int on_device;                /* 1: the pointers above are device pointers of the context's device */
    /* filled by the engine */
    int row, col;
    int n_slices;
    double interval_x, interval_y;
    double total_intensity;
} ms_output;

typedef struct ms_ctx ms_ctx;

/* ---- library and context ------------------------------------------------ */
const char* ms_version(void);
int ms_abi_version(void);
/* Fill `p` with this engine's defaults (multislice_params constructor). */
void ms_default_params(ms_params* p);
/* multislice_params::validate_parameters (simulator.cu:15, :25, :38). */
ms_status ms_validate_params(const ms_params* p);
/* Creates a context on `device` (run_simu: cudaSetDevice, single_simulator.cuh:208-211). */
ms_status ms_create(ms_ctx** ctx, int device);
ms_status ms_destroy(ms_ctx* ctx);
const char* ms_last_error(const ms_ctx* ctx);
/* Run on a caller stream (a cudaStream_t) instead of the context's own; NULL restores the own stream. */
ms_status ms_set_stream(ms_ctx* ctx, void* cuda_stream);
void* ms_get_stream(ms_ctx* ctx);
/* Device time (ms) of the last simulate call, measured with CUDA events on the context stream. */
double ms_last_device_ms(const ms_ctx* ctx);
/* Number of this library's kernels launched by the last call (kernels replayed from a
 * captured CUDA graph included). */
int64_t ms_last_launch_count(const ms_ctx* ctx);
/* Probes per batch used by the last STEM call: the autotuner's choice when probe_batch is 0.
 * No reference counterpart (the reference's batch is the fixed c_Probe_Batch,
 * multislice_params_dev.cuh:92-108). */
int ms_last_probe_batch(const ms_ctx* ctx);
/* Enables (1, the default) or disables (0) replaying each STEM probe batch from a captured
 * CUDA graph.  Disabled, every launch is issued directly; the results are identical. */
ms_status ms_set_graphs(ms_ctx* ctx, int enable);
/* Kernel form of the hot slice passes: 0 (default) the classic kernels, one block per tile
 * of rows or columns, launched slice by slice for CBED / TEM / STEM, while an uneven batch's grid
 * groups run in the persistent slice engine (form 2); 3 the classic kernels everywhere, uneven
 * batches included; 1 the persistent pipelined kernels
 * (one block per SM walking the work items, the next item's wave prefetched while the
 * current one is transformed) for grids of 128..1024 points per axis; 2 the persistent slice
 * engine: on square grids, every slice of a CBED / TEM / STEM batch or of an uneven batch's
 * grid group runs in one launch whose blocks take row and column work items in slice order
 * and wait (bounded) for each wave's earlier items through per-wave slice counters.  All
 * forms compute the same operations (results agree to float rounding); the choice only
 * changes speed.  No reference counterpart (the reference's passes are cuFFT plans). */
ms_status ms_set_pass_kernels(ms_ctx* ctx, int variant);   /* 0..3 */
/* Tile shape of the classic hot passes (the row step on the transmission store and the column
 * step): -1 (default) autotuned per grid and batch size; otherwise a bit mask, bit 0 narrow rows
 * (one warp of rows per block, twiddles from L1), bit 1 narrow columns (four columns per block),
 * bit 2 one warp per column (1024-point columns; swizzled tile and transposed propagator; takes
 * precedence over bit 1): 0 wide tiles (blocks of 8..16 rows or columns), 1 narrow rows, 2 narrow
 * columns, 3 both, 4 warp columns, 5 warp columns and narrow rows.  Narrow
 * tiles spread batches too small to fill the GPU over every SM.  The autotuner times the four
 * shapes on the call's own data the first time a grid and batch size are seen.  All shapes
 * compute the same operations bit for bit.  No reference counterpart (the reference's FFTs are
 * cuFFT plans). */
ms_status ms_set_tile_shape(ms_ctx* ctx, int shape);
/* How CBED / TEM / STEM calls keep their slices between the potential kernel and the slice loop:
 * 1 (default) as the transmission function t = exp(iσV) (FP32 complex, formed once per pixel in
 * the potential kernel), 0 as σV (FP32, t formed in the row step from the same table).  Both give
 * the same values; the choice trades the store's size and traffic against row-step arithmetic. */
ms_status ms_set_transmission_store(ms_ctx* ctx, int enable);
/* Tile shape (the bit mask above) of the last CBED / TEM / STEM call's hot passes. */
int ms_last_tile_shape(const ms_ctx* ctx);
/* JSON file that keeps the autotuner's choices (probe batch, tile shape) across contexts and
 * processes, keyed by device, grid and batch size; entries already in the file are loaded now.
 * NULL or "" keeps the choices in the context only (the default).  A missing or unreadable file
 * starts empty; an unwritable one only loses the persistence. */
ms_status ms_set_tune_cache(ms_ctx* ctx, const char* path);
/* Order of the projected-potential work in the TEM, ED, CBED and thickness simulations:
 * 0 (default) every slice's potential before the slice loop, on the context stream; 1 the
 * potentials in 16-slice chunks, all but the first on a side stream while the slice passes of
 * earlier slices run.  The results are identical.  The overlapped order competes with the
 * slice passes for the SMs (a pass block needs the registers of half an SM), which makes a
 * step slower than the serial order on some runs.  No reference counterpart (the reference
 * generates each slice's potential just before its transmission, transmission_function.cuh:82-134). */
ms_status ms_set_potential_overlap(ms_ctx* ctx, int enable);

/* Host-side fault injection for tests of the failure paths (no reference counterpart).
 * MS_INJECT_WAIT_TIMEOUT makes the column passes of the TEM/ED/CBED loop wait for a shared-memory
 * tile that is never completed: the bounded device-side wait runs out after about a millisecond,
 * the kernel records it and returns, and the call fails with MS_ERR_TIMEOUT; the context stays
 * usable.  MS_INJECT_ALLOC_FAIL makes every device allocation the context would make fail, as a
 * cudaMalloc that ran out of memory: the call fails with MS_ERR_OUT_OF_MEMORY and the context
 * stays usable.  MS_INJECT_NONE (0) switches injection off. */
enum { MS_INJECT_NONE = 0, MS_INJECT_WAIT_TIMEOUT = 1, MS_INJECT_ALLOC_FAIL = 2 };
ms_status ms_set_fault_injection(ms_ctx* ctx, int what);

/* Per-kernel timing (no reference counterpart: the reference has no tracing).  While enabled,
 * every fused pass and potential launch is bracketed by CUDA events on the context stream;
 * ms_profile_get returns the launches and summed device time of one kernel class
 * since the last reset: "row", "col" (forward slice passes), "potential", "probe", and the
 * adjoint's "row_store" (forward row pass that keeps the transmitted wave), "row_adj",
 * "col_adj", "seed", "grad_probe". */
ms_status ms_set_profiling(ms_ctx* ctx, int enable);
ms_status ms_profile_reset(ms_ctx* ctx);
ms_status ms_profile_get(const ms_ctx* ctx, const char* kernel, int64_t* launches, double* total_ms);

/* ---- physics (missing host headers, re-derived) ---------------------------- */
/* Relativistic wavelength (A), interaction constant sigma (rad/(V*A)), factor gamma. */
ms_status ms_physics(double E0_kV, double* lambda, double* sigma, double* gamma);

/* ---- simulator entry points ---------------------------------------------- */
/* mulSimulator::executionTEM (simulator.cu:8-19): HRTEM image or ED pattern. */
ms_status ms_simulate_tem(ms_ctx* ctx, const ms_params* p, const ms_atoms* atoms, ms_output* out);
/* Defocus series of HRTEM images from one multislice run: the exit waves are imaged through the
 * objective lens at C10 + defocus[i] for i < n_defocus, each image summed over the phonon
 * configurations (apply_CTF_kernel_batch, device_kernels.cuh:469-503, which adds defocus[i] g^2 to
 * the lens phase of a batch of copies of the exit wave; the reference defines it without a
 * driver, so the batch is exposed here as its own entry point).  Coherent CTF only
 * (illumination_model coherent).  out->image_intensity (data_record intensity) or
 * out->image_real / out->image_imag (data_record wave) hold n_defocus*ny*nx floats, laid out
 * [defocus][row][col]. */
ms_status ms_simulate_tem_defocus_series(ms_ctx* ctx, const ms_params* p, const ms_atoms* atoms, int n_defocus,
                                         const double* defocus, ms_output* out);
/* mulSimulator::executionCBED (simulator.cu:20-30): CBED pattern. */
ms_status ms_simulate_cbed(ms_ctx* ctx, const ms_params* p, const ms_atoms* atoms, ms_output* out);
/* mulSimulator::executionSTEM (simulator.cu:31-49): annular-detector STEM image. */
ms_status ms_simulate_stem(ms_ctx* ctx, const ms_params* p, const ms_atoms* atoms, ms_output* out);
/* Thickness_simulator::Thickness_multiGPU (thickness_simulator.cuh:96-118): filtered intensity after every slice. */
ms_status ms_simulate_thickness(ms_ctx* ctx, const ms_params* p, const ms_atoms* atoms, ms_output* out);

/* ---- specimen and slicing (Specimen / Slice_Generator) ---------------------- */
/* Displaced coordinates of configuration `conf` (1-based, as the reference's phonon loop,
 * single_simulator.cuh:60-75); conf 0 returns the undisplaced atoms. */
ms_status ms_displace_atoms(const ms_params* p, const ms_atoms* atoms, int conf,
                            float* x_out, float* y_out, float* z_out);
/* Slice_Generator::calculate (slice_generator.hpp:48-168) on configuration `conf`:
 * `bounds` gets n_slices+1 plane positions; `atom_slice` gets each atom's slice index
 * (-1 when the atom lies outside every slice).  Either pointer may be NULL. */
ms_status ms_build_slices(const ms_params* p, const ms_atoms* atoms, int conf,
                          int* n_slices, float* bounds, int bounds_capacity, int* atom_slice);
/* Crystal slab builder: the unit cell (nb basis atoms at fractional coordinates) repeated
 * na x nb_rep x nc times.  With x == NULL only the atom count is returned in *n_out. */
ms_status ms_build_crystal(int n_basis, const int* basis_Z, const double* basis_frac_xyz,
                           double a, double b, double c, int na, int nb_rep, int nc,
                           float sigma, float occ,
                           int64_t* n_out, int* Z, float* x, float* y, float* z, float* sigma_out, float* occ_out);

/* ---- projected potential (Projected_Potential::generate_potential_by_slice,
 *      projected_potential.cuh:47-92, on the device kernel) ------------------ */
/* Writes sigma-scaled projected potentials (Vr_factor * V_z, rad) of every slice of
 * configuration `conf` into V_out [n_slices][ny][nx]; `capacity` is in floats. */
ms_status ms_projected_potential(ms_ctx* ctx, const ms_params* p, const ms_atoms* atoms, int conf,
                                 float* V_out, int64_t capacity, int V_on_device, int* n_slices);

/* ---- slice loop on caller potentials (wave_modulation_batch, wave_function.cuh:74-87) ---- */
/* Runs a convergent probe at each of `n_probe` positions (probe_xy = x0,y0,x1,y1,... in A)
 * through slices with the given phase arrays V[n_slices][ny][nx] (rad; t = exp(i V)), and
 * writes the annular-detector intensities I[n_probe][n_det].  z_init is the defocus shift
 * of the probe (slice_middle_z(0), wave_function.cuh:56). */
ms_status ms_stem_forward_potential(ms_ctx* ctx, const ms_params* p, const float* V, int n_slices,
                                    int V_on_device, double z_init, const double* probe_xy, int n_probe,
                                    float* I_out);
/* The same computation as ms_stem_forward_potential for callers that cannot let a library
 * allocate device memory (an application whose memory manager owns every allocation, or a
 * loop that must not pay cudaMalloc's implicit synchronisation).  No reference counterpart:
 * the reference allocates per call.  It allocates nothing and needs no context: V (device,
 * [n_slices][ny][nx]) and I_out (device, [n_probe][n_det]) are the caller's device memory,
 * probe_xy is host memory, and the work runs on `cuda_stream` (NULL = legacy default stream)
 * of the current device.  All scratch -- waves, twiddles, propagator factors, detector
 * partial sums -- lives in one fixed array of about 34 MiB held by every GPU that loads the
 * library until exit; grids with nx*ny*8 bytes above 32 MiB (larger than 2048 x 2048) are
 * rejected with MS_ERR_UNSUPPORTED.  The first call on each device looks the array up (again
 * after the device's CUDA context changes, e.g. after cudaDeviceReset); that first call should
 * come before any stream capture.  The call uploads
 * probe positions from host memory and synchronises the stream after every probe batch, so it
 * blocks the host until its results are in I_out.  All calls share the array, so calls that
 * overlap on the GPU race and must be serialised.  Errors are read with ms_last_error(NULL),
 * which a successful call clears. */
ms_status ms_stem_forward_potential_noalloc(void* cuda_stream, const ms_params* p, const float* V, int n_slices,
                                            double z_init, const double* probe_xy, int n_probe, float* I_out);
/* Adjoint of ms_stem_forward_potential for the loss L = sum_{probe,det} (I - target)^2:
 * loss, dL/dV [n_slices][ny][nx] (summed over probes) and dL/dC10, dL/dC30 of the condenser
 * lens (C10 includes z_init; C30 is Cs).  The waves are checkpointed every p->ckpt_interval
 * slices and each segment's transmitted waves are recomputed from its checkpoint.  V and
 * dL_dV are device pointers when V_on_device is 1, host pointers otherwise; probe_xy and
 * target ([n_probe][n_det]) are host memory.  dL/dV is summed over probes in a fixed order, so
 * repeated calls give the same bits.  No reference counterpart: the reference has no
 * differentiable path. */
ms_status ms_stem_backward(ms_ctx* ctx, const ms_params* p, const float* V, int n_slices, int V_on_device,
                           double z_init, const double* probe_xy, int n_probe, const float* target,
                           double* loss, float* dL_dV, double* dL_dC10, double* dL_dC30);

/* ---- uneven batched workload (no reference counterpart: the reference runs one
 *      simulation per call) ---------------------------------------------------- */
/* Runs n independent CBED/STEM simulations of possibly different grid sizes in one
 * scheduled launch sequence.  latency_ms (may be NULL) gets each instance's completion
 * time relative to the start of the call, measured on the device. */
ms_status ms_simulate_many(ms_ctx* ctx, int n, const ms_params* params, const ms_atoms* atoms,
                           ms_output* outs, double* latency_ms);

#ifdef __cplusplus
}
#endif
#endif /* CUDAEM_B200_H */
