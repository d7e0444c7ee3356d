/*
 * rtw.h - C ABI of librtw_b200.so, the B200 geodesic spectral ray tracer.
 *
 * The library integrates camera rays backwards through a curved spacetime
 * with an adaptive Dormand-Prince RK45 step loop, co-integrating the
 * "slow-light" radiative transfer (invariant intensity I_nu/nu^3 and optical
 * depth tau_nu per spectral bin), and reduces each ray's spectrum to linear
 * CIE XYZ. It is a drop-in for the integrator behind the reference's render
 * call:
 *
 *   gen_image(; camera_pos, camera_dir, speed, camera_point, x_pix, max_steps,
 *              colors, returnrays, tolerance, max_dt_scale, fov_hor, fov_vert,
 *              print_num_pix, ray_bundles)
 *     main/Iterators/LttM/LttM.jl:104-209 (CPU), main/Iterators/5P/5P.jl:135-282 (GPU)
 *
 * and for the per-scene ".source" plugin contract (metric, Christoffel
 * symbols, singularity guards, emitter, step cap, termination), e.g.
 *   main/Kerr.source/source_geometry.jl:55-315, main/Kerr.source/source_model.jl:9-189.
 *
 * Every entry point takes plain pointers and sizes; no C++ or torch types
 * cross this boundary. All functions return rtw_status and never abort the
 * process; the text of the last error of a context is in rtw_last_error().
 */
#ifndef RTW_H
#define RTW_H

#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define RTW_ABI_VERSION 7
/* Largest number of spectral bins (reference `colors`) one render takes. */
#define RTW_MAX_BINS 128
/* Largest number of frames (cameras) one batched render takes. */
#define RTW_MAX_FRAMES 4096
/* Doubles per record of the step trace (rtw_outputs.trace). */
#define RTW_TRACE_FIELDS 15

typedef enum rtw_status {
    RTW_OK = 0,
    RTW_ERR_INVALID_CAMERA = 1, /* camera on a coordinate singularity
                                   (reference: is_singularity, 5P.jl:140-143) */
    RTW_ERR_INVALID_PARAM = 2,  /* a size, pointer or parameter out of range   */
    RTW_ERR_CUDA = 3,           /* a CUDA runtime call failed                  */
    RTW_ERR_ITER_LIMIT = 4,     /* a device loop hit its iteration cap         */
    RTW_ERR_NAN = 5,            /* non-finite values in the initial data       */
    RTW_ERR_NO_DEVICE = 6,      /* no CUDA device / wrong architecture         */
    RTW_ERR_UNSUPPORTED = 7,    /* feature not built (e.g. ray bundles)        */
    RTW_ERR_OOM = 8             /* device allocation failed                    */
} rtw_status;

/* Scene kinds: the ".source" folders of the reference that are on the hot path,
 * with their constants turned into runtime parameters (rtw_scene). */
typedef enum rtw_scene_kind {
    /* Minkowski_Sphere_Spherical.source: flat space in (t,r,theta,phi),
       emitting sphere r <= r_out. */
    RTW_SCENE_MINKOWSKI_SPHERE = 0,
    /* Schwarzschild_Simple_Disk_Spherical.source: wedge disk
       r_in <= r <= r_out, theta_lo <= theta <= theta_hi. */
    RTW_SCENE_SCHWARZSCHILD_DISK = 1,
    /* Kerr.source (Boyer-Lindquist): wedge disk with Keplerian emitter,
       ZAMO outside it; spin is a runtime value. */
    RTW_SCENE_KERR_DISK = 2,
    /* Kerr with a thickened, optically thin disk: rho = (r/r0)^-2
       exp(-z^2 / 2 (h r)^2), alpha = a_nu * rho, j = alpha B_nu(T),
       T = temperature (r/r0)^t_index, for r_in <= r <= r_out. */
    RTW_SCENE_KERR_THICK_DISK = 3,
    /* Kerr with an optically thin-to-thick thermal synchrotron torus (no
       reference counterpart; a new .source emitter behind the same RT slot
       contract, integrators_LttM.jl:33-42). With x = r / r_in and
       z = r cos(theta):
         n_e   = n_e0 x^rho_index exp(-z^2 / 2 (rho_h r)^2)
         B     = b_0 x^b_index          (toroidal, fluid frame)
         Theta = theta_e0 x^t_index     (kT_e / m_e c^2)
       tapered by exp(-((r_in - r)/edge_in)^2) inside r_in and by
       exp(-((r - r_out)/edge_out)^2) outside r_out (zero beyond 4 widths);
       Keplerian 4-velocity; thermal synchrotron j_nu from the Leung, Gammie
       & Noble (2011) fit, alpha_nu = j_nu / B_nu(T_e). Per-bin tau. Only
       the FSAL integrator. */
    RTW_SCENE_KERR_SYNCHRO_TORUS = 4,
    /* Powehi.source, the reference's M87* model: Kerr (spin), a blackbody
       wedge disk (r_in..r_out, theta_lo..theta_hi, a_nu, temperature) and a
       rotating conical jet beyond r = 10 within 5 deg of the axis (Lorentz
       factor 1.2 -> 10 over r = 10..75) radiating power-law synchrotron
       (p = 2.5, gamma 30..1e9, anisotropy fit) in a global field B^phi = b_0,
       electron density n_e0 (m^-3), map scale length_cm
       (source_model.jl:7-317). Per-bin tau; both integrators. */
    RTW_SCENE_KERR_POWEHI = 5,
    /* Synchro_Test.source, the reference's flat-space synchrotron test:
       Minkowski space in Cartesian coordinates (t, x, y, z) (camera
       position and ray states are Cartesian), a static cylinder x^2 + y^2 <=
       r_out^2 around the z axis in a uniform field B^z = b_0 (gauss),
       radiating power-law synchrotron (p = 2.5, gamma 30..1e9, anisotropy
       fit) with n_e0 (m^-3) and map scale length_cm; rays end beyond
       |x| = escape_radius (source_geometry.jl:7-88, source_model.jl:7-278).
       Per-bin tau; both integrators. */
    RTW_SCENE_SYNCHRO_TEST = 6,
    /* Wormhole.source, the reference's Dneg wormhole: coordinates (t, l,
       theta, phi), metric -dt^2 + dl^2 + r(l)^2 dOmega^2 with throat radius
       r_in, half-length edge_in and lensing width edge_out (Interstellar's:
       1, 0.005, 0.05); empty space; rays end beyond r(l) = escape_radius or
       phi > winding_limit (source_geometry.jl:7-205, source_model.jl:54-147).
       Both integrators. */
    RTW_SCENE_WORMHOLE = 7,
    /* Minkowski_Sphere_Cartesian.source ("minkowski_t,x,y,z_sphere"): flat
       space in Cartesian (t, x, y, z), a static blackbody sphere of radius
       r_out at temperature (5778 K) with a_nu = a_nu (1 per map unit, so
       optically thin: tau <= 2) in front of skybox[0], which every ray adds at
       its end; rays end beyond |x| = escape_radius (source_geometry.jl:7-82,
       source_model.jl:8-431). Both integrators. */
    RTW_SCENE_MINKOWSKI_CART_SPHERE = 8,
    /* Kerr with a thermal bremsstrahlung torus: the fluid of
       RTW_SCENE_KERR_SYNCHRO_TORUS (n_e, Theta_e, tapers, Keplerian
       4-velocity; no field), radiating free-free emission
         j_nu = C n_e^2 Theta_e^(-1/2) exp(-u) g_ff(gamma^2, u),
         u = h nu / (Theta_e m_e c^2), gamma^2 = Ry / (Theta_e m_e c^2),
       C = 7.089314638783696e-44 erg cm^3 s^-1 Hz^-1 sr^-1 (C_Yar_cgs,
       emission_functions.jl:19), alpha_nu = j_nu / B_nu(T_e). g_ff is the
       reference's gaunt_ei_therm_van_Hoof (emission_functions.jl:54-78): a
       bilinear lookup in the van Hoof (2014) merged Gaunt-factor table that
       the caller passes as rtw_render_params.gaunt_lut, in Float32 with its
       index offsets and its fallback 1.2 outside the table. No scene of the
       reference calls that function. Per-bin tau; both integrators. */
    RTW_SCENE_KERR_BREMS_TORUS = 9
} rtw_scene_kind;

/* How a ray ended. The reference's calc_terminate (e.g. Kerr.source/
 * source_model.jl:168-182) returns only a Bool; the class is the first of its
 * predicates that holds, in the reference's order. */
typedef enum rtw_term_class {
    RTW_CLASS_NONE = 0,     /* not traced                                       */
    RTW_CLASS_ESCAPE = 1,   /* r > escape_radius                                */
    RTW_CLASS_HORIZON = 2,  /* r <= (1 + 10 tol) r_horizon                      */
    RTW_CLASS_THICK = 3,    /* every tau slot >= -log(tol): hit disk / body      */
    RTW_CLASS_WINDING = 4,  /* phi > winding_limit (8 pi)                       */
    RTW_CLASS_MAXSTEPS = 5, /* step_count >= max_steps (checked first)          */
    RTW_CLASS_NAN = 6       /* the final geodesic state is not finite           */
} rtw_term_class;

typedef enum rtw_precision {
    RTW_PREC_FP64 = 0,  /* every stage, RHS and RT update in FP64             */
    RTW_PREC_MIXED = 1, /* FP64 state + controller, FP32 stages/RHS/RT with
                           Kahan-compensated intensities, per-ray FP64 stages
                           near the horizon and the polar axis               */
    RTW_PREC_FP64_PLAIN = 2 /* the plain FP64 GPU path, the baseline: one thread
                           per pixel over a grid, the reference's full state of
                           8 + 2N components with every bin's coefficients in
                           every right-hand side (ray_kernel / integrate_ray,
                           LttM.jl:11-80; calc_ray_derivative!,
                           integrators_LttM.jl:9-48), no warp cooperation  */
} rtw_precision;

typedef enum rtw_integrator {
    /* Reference semantics (integrators_LttM.jl:147-150,199,219): the next
       step's k1 is the weighted average slope sum(b_i k_i), not f(y). */
    RTW_DP45_REF_COMPAT = 0,
    /* Textbook FSAL Dormand-Prince: the next step's k1 is k7 = f(y). */
    RTW_DP45_FSAL = 1
} rtw_integrator;

/* Scene parameters. Fields a scene kind does not use are ignored.
 * rtw_scene_default() fills the reference's values for a kind. */
typedef struct rtw_scene {
    int32_t kind;           /* rtw_scene_kind */
    int32_t ref_precision;  /* 1: Kerr Christoffel symbols in FP32 as the
                               reference's CPU path computes them
                               (Kerr.source/source_geometry.jl:196-197) */
    double mass;            /* M (G = c = 1); reference M = 1 */
    double spin;            /* Kerr a (|a| < M); reference 0.998 */
    double r_in;            /* emitter inner radius (disk) */
    double r_out;           /* emitter outer radius (disk) / sphere radius */
    double theta_lo;        /* wedge lower polar angle */
    double theta_hi;        /* wedge upper polar angle */
    double temperature;     /* blackbody temperature, K */
    double a_nu;            /* absorption coefficient, 1 / map unit */
    double escape_radius;   /* reference: 100 */
    double winding_limit;   /* reference: 8 pi */
    double rho_r0;          /* thick disk: reference radius r0 (6 M) */
    double rho_h;           /* thick disk: scale height / r (0.1) */
    double rho_index;       /* thick disk: density power law (-2) */
    double t_index;         /* thick disk: temperature power law (-0.75) */
    /* synchrotron torus (RTW_SCENE_KERR_SYNCHRO_TORUS); r_in is the torus
       inner radius, r_out the start of the outer taper, rho_h the Gaussian
       scale height / r, rho_index / t_index the n_e / Theta_e power laws */
    double n_e0;            /* electron density at r_in, cm^-3 */
    double b_0;             /* magnetic field at r_in, gauss */
    double theta_e0;        /* dimensionless electron temperature at r_in */
    double b_index;         /* field power law */
    double edge_in;         /* inner taper width, M */
    double edge_out;        /* outer taper width, M */
    double length_cm;       /* GM/c^2 in cm (the map unit) */
} rtw_scene;

/* One camera (= one frame of a batch). Mirrors the camera keywords of
 * gen_image and initialize_camera (initialization.jl:190-331). */
typedef struct rtw_camera {
    double position[4];     /* camera_pos: (t, r, theta, phi) */
    double direction[2];    /* camera_dir: direction of the camera's
                               3-velocity relative to the local tetrad */
    double speed;           /* speed (beta), |beta| < 1 */
    double pointing[3];     /* camera_point: roll, pitch, yaw */
    int32_t x_pix;          /* x_pix: horizontal pixels */
    int32_t y_pix;          /* out: round(x_pix * tan(fov_vert/2) / tan(fov_hor/2)) */
    double fov_hor;         /* degrees */
    double fov_vert;        /* degrees */
    double tolerance;       /* abs_tol = rel_tol for every state component */
    int64_t max_steps;      /* step-attempt cap per ray */
    /* window: render only pixels [win_x0, win_x0 + win_w) x [win_y0, win_y0 +
       win_h) of the x_pix x y_pix image (win_w = win_h = 0: the whole image).
       The window's rays are those of the whole image; its outputs are its own
       pixels, row-major. Used to split one frame over GPUs in interleaved
       tiles. No counterpart in the reference (one image per call). */
    int32_t win_x0, win_y0, win_w, win_h;
} rtw_camera;

typedef struct rtw_render_params {
    int32_t n_colors;           /* number of spectral bins, 1..RTW_MAX_BINS */
    int32_t precision;          /* rtw_precision */
    const double* colors_nm;    /* [n_colors] wavelengths in nm (reference
                                   `colors`); host memory */
    double max_dt_scale;        /* reference max_dt_scale (default 0.1) */
    int32_t integrator;         /* rtw_integrator */
    int32_t ray_bundles;        /* 1: Gaussian ray-bundle lookup of the skyboxes
                                   (RTW_SCENE_WORMHOLE, RTW_SCENE_MINKOWSKI_CART_SPHERE;
                                   other scenes return RTW_ERR_UNSUPPORTED); as in
                                   the reference, no opacity stop then */
    double promote_dr;          /* MIXED: FP64 stages while r - r_horizon < promote_dr M
                                   (0: default 1e-3; < 0: never) */
    double promote_sin;         /* MIXED: FP64 stages while sin(theta) < promote_sin
                                   (0: default 2e-3 in the trace kernel, 1e-2 in
                                   the per-bin kernels (Powehi 0.1); < 0: never) */
    int32_t block_warps;        /* warps per CTA, 1..4 (0: default 4) */
    int32_t ctas_per_sm;        /* resident CTAs per SM (0: default) */
    void* stream;               /* cudaStream_t to run on; NULL: the context's
                                   stream, and rtw_render returns when done */
    int32_t pixel_order;        /* 0: row order; 1: 8x4 tiles (internal order,
                                   outputs are always row order) */
    int32_t refill_min;         /* compaction interval: a warp takes new rays once
                                   at least this many of its 32 lanes are free
                                   (or all are); 0: default 1 */
    int64_t trace_ray;          /* global pixel index whose step attempts are
                                   recorded in rtw_outputs.trace; -1: none */
    int32_t autotune;           /* 1: block_warps and refill_min (where 0) come
                                   from a per-context autotuner that times the
                                   candidates once per scene kind, precision,
                                   bin count and integrator, on the first
                                   camera at up to 768 pixels wide */
    int32_t graph;              /* 1: the launch sequence (frame table upload,
                                   counter reset, kernel) is captured once in a
                                   CUDA graph and replayed while the launch
                                   parameters match; cameras may change */
    /* RTW_SCENE_WORMHOLE: the two skyboxes (skybox[0] beyond the throat's
       positive-l side, skybox[1] beyond its negative side), each a cube map in
       the reference's cross layout: skybox_h[k] pixels per face edge, 3 h rows
       x 4 h columns of (R, G, B) float32 in [0, 1], row 0 at the top (the
       PNGs the reference loads in load_textures; NULL: no skybox). Host
       memory. A ray that ends beyond r(l) = 50 adds the texel it points at,
       as the reference's skybox_handling! without ray bundles does, or, with
       ray_bundles = 1, the texels within a Gaussian footprint of the pixel's
       ray bundle (up to 21 x 21 texels, across face edges), as its
       calc_skybox_I_nu_beam! does (Wormhole.source/source_model.jl:150-443).
       RTW_SCENE_MINKOWSKI_CART_SPHERE: skybox[0] only, added at the end of
       every ray (Minkowski_Sphere_Cartesian.source/source_model.jl:175-431). */
    const float* skybox[2];
    int32_t skybox_h[2];
    /* RTW_SCENE_KERR_BREMS_TORUS: the van Hoof merged Gaunt-factor table
       (Main/Gaunt_Factors/gauntff_merged_Z01.dat without its 42 header lines):
       RTW_GAUNT_ROWS rows of constant log10 u (-16, -15.8, ...) by
       RTW_GAUNT_COLS columns of constant log10 gamma^2 (-6, -5.8, ...),
       row-major float32, host memory (the reference's Gaunt_LUT[i, j] is
       gaunt_lut[(i - 1) * RTW_GAUNT_COLS + (j - 1)]). Required for that scene. */
    const float* gaunt_lut;
    /* FP32-mixed trace kernel (kinds 0-3): 0 (default) hands each ray that
       comes within promote_dr of the horizon (from where it falls in, with
       FP64 stages) to a second pass of the kernel that traces such rays in
       whole warps (the results are the same bit for bit); -1 keeps every ray
       in its lane, with FP64 stages there. */
    int32_t tail_pass;
} rtw_render_params;

#define RTW_GAUNT_ROWS 146
#define RTW_GAUNT_COLS 81

/* Output buffers, owned by the caller. Pixel p of frame f is at
 * frame_offset(f) + i + x_pix * j, with i the horizontal index (reference
 * canvas index i, initialization.jl:213-214) and j the vertical one. NULL
 * pointers are skipped. */
typedef struct rtw_outputs {
    float* xyz;             /* [P][3] linear CIE XYZ (color_theory.jl:96-108
                               before the xyY conversion) */
    uint8_t* term_class;    /* [P] rtw_term_class */
    uint32_t* steps;        /* [P] step attempts (incl. rejected) */
    float* spectrum;        /* [P][n_colors] final invariant intensity
                               I_nu/nu^3 per bin (reference Ray[9+2c]) */
    double* final_state;    /* [P][8] final (t,r,theta,phi,k^t,k^r,k^theta,k^phi) */
    float* tau;             /* [P] final optical depth (every tau slot of the
                               reference's state holds this value: the emitters
                               are grey) */
    int32_t on_device;      /* 1: device pointers; 0: host pointers */
    int32_t trace_capacity; /* records that fit in trace */
    double* trace;          /* [trace_capacity][RTW_TRACE_FIELDS] step attempts
                               of params->trace_ray: step, the step size of the
                               next attempt, accepted,
                               promoted, escaped, err^2 (unnormalised), then
                               the state t, r, theta, phi, k^t, k^r, k^theta,
                               k^phi, tau after the attempt; unused records
                               are NaN */
} rtw_outputs;

typedef struct rtw_stats {
    uint64_t rays;              /* rays traced by the last render */
    uint64_t step_attempts;     /* DP45 step attempts, all rays */
    uint64_t rejected_steps;    /* rejected attempts, all rays */
    uint64_t promoted_steps;    /* MIXED: attempts run with FP64 stages */
    uint64_t spectral_steps;    /* attempts whose spectral slots were updated */
    uint64_t emitting_steps;    /* attempts with emission in some stage */
    uint64_t escape_substeps;   /* polar Euler sub-steps */
    uint64_t nan_rays;          /* rays of class RTW_CLASS_NAN */
    double kernel_ms;           /* device time of the trace kernel */
    double total_ms;            /* device time of the whole render call */
    uint64_t phase_cycles[4];   /* builds with RTW_PHASE_CLOCKS only (else 0): SM
                                   cycles summed over warps in refill, geodesic,
                                   spectral, commit/epilogue */
    int32_t grid;               /* launch shape used: CTAs */
    int32_t block_warps;        /*   warps per CTA */
    int32_t refill_min;         /*   compaction interval */
    int32_t graph_replayed;     /* 1: the render replayed a captured graph */
    uint64_t tail_rays;         /* FP32-mixed trace kernel: rays finished by the
                                   FP64 tail pass */
    int32_t launches;           /* this library's kernel launches in the last
                                   render call (2 for an FP32-mixed trace render
                                   with its tail pass) */
    int32_t reserved0;
} rtw_stats;

/* Algorithmic operation counts of the trace kernel's arithmetic for one scene
 * kind (add/sub/mul = 1 flop, an FMA = 2; div/sqrt/exp = 1 flop + 1 MUFU op;
 * sincos/pow = 2 + 2), counted by running the kernel's own formulas on the
 * host with a counting scalar. */
typedef struct rtw_op_counts {
    double rhs_vacuum;          /* one right-hand side outside every emitter */
    double rhs_vacuum_mufu;
    double rhs_emit;            /* one right-hand side inside the emitter    */
    double rhs_emit_mufu;
    double step_overhead;       /* one DP45 attempt without its 6 right-hand
                                   sides: stage sums, error norm, controller */
    double step_overhead_mufu;
    double bin_step;            /* one spectral bin of one updated attempt   */
    double bin_step_mufu;
} rtw_op_counts;

typedef struct rtw_ctx rtw_ctx;

/* Creates a context on CUDA device `device` (its own stream, cached device
 * buffers). Replaces the CuArray set-up of 5P.jl:177-198. */
rtw_status rtw_create(rtw_ctx** out, int32_t device);
/* Frees the context and its device buffers. NULL is accepted. */
void rtw_destroy(rtw_ctx* ctx);
/* Text of the context's last error ("" if none); valid until the next call. */
const char* rtw_last_error(const rtw_ctx* ctx);
/* ABI version (RTW_ABI_VERSION) of the loaded library. */
int32_t rtw_abi_version(void);

/* Fills the reference's constants for a scene kind (Kerr.source,
 * Schwarzschild_Simple_Disk_Spherical.source, Minkowski_Sphere_Spherical.source
 * source_model.jl / source_geometry.jl constants). */
rtw_status rtw_scene_default(int32_t kind, rtw_scene* out);

/* Sets cam->y_pix = round(x_pix tan(fov_vert/2) / tan(fov_hor/2)) with ties to
 * even (initialization.jl:197-200) and returns the count of pixels the camera
 * renders in *n_pix (the image's, or its window's). */
rtw_status rtw_camera_pixels(rtw_camera* cam, int64_t* n_pix);

/* Host FP64 initial data of one camera, the reference's initialize_camera
 * (initialization.jl:190-331): rays_out[P][8] = (x^mu, k^mu) per pixel,
 * pixel order as in rtw_outputs. The spectral slots start at zero. */
rtw_status rtw_camera_rays(const rtw_scene* scene, const rtw_camera* cam,
                           double* rays_out, int64_t n_pix);

/* Trapezoid CIE weights for the bins (precompute_CIE_weights,
 * color_theory.jl:79-91, generalised to non-uniform spacing) and the
 * per-bin factor nu^3 c / lambda^2 of ray_to_I_lambda (color_theory.jl:73). */
rtw_status rtw_cie_weights(const double* colors_nm, int32_t n_colors,
                           double* w_x, double* w_y, double* w_z, double* i_lambda_factor);

/* Renders n_cams frames of one scene in one persistent launch. Replaces the
 * integrate + colour part of gen_image (5P.jl:158-249, LttM.jl:141-176).
 * With params->stream == NULL the call is synchronous. */
rtw_status rtw_render(rtw_ctx* ctx, const rtw_scene* scene,
                      const rtw_camera* cams, int32_t n_cams,
                      const rtw_render_params* params, rtw_outputs* out);

/* Counters and device times of the last rtw_render on this context
 * (synchronises the context's stream). */
rtw_status rtw_get_stats(rtw_ctx* ctx, rtw_stats* out);

/* Per-frame timing of the last rtw_render on this context, from the device's
 * global nanosecond timer: done_ms[f] = time from the start of the batch's
 * first ray to the end of frame f's last ray; span_ms[f] = from frame f's
 * first ray start to its last ray end (either may be NULL). n_frames must be
 * the n_cams of that render. No counterpart in the reference (one frame per
 * gen_image call). */
rtw_status rtw_get_frame_times(rtw_ctx* ctx, int32_t n_frames, double* done_ms, double* span_ms);

/* ---- differentiable synchrotron torus: discrete adjoint -------------------
 * The loss is L = sum over pixels p and bins c of (I_pc - target_pc)^2 with
 * I the final invariant intensity (the spectrum output). Parameters, in this
 * order: spin a, camera inclination (position[2], rad), n_e0, b_0, theta_e0.
 * The gradient is that of the discrete FSAL Dormand-Prince map along each
 * ray's accepted steps (step sizes held fixed, as in any discrete adjoint of an
 * adaptive integrator), reversed from states checkpointed every
 * checkpoint_every accepted steps and recomputed in FP64 in between. The
 * camera initial data enter through their derivative in a and the
 * inclination (a central difference of the FP64 camera transform, which is
 * linear in the transform matrix). No counterpart in the reference (it has
 * no derivatives); it backs a ChainRulesCore rrule of gen_image. */
#define RTW_ADJOINT_PARAMS 5

typedef struct rtw_adjoint_params {
    const float* target;        /* [P][n_colors] target spectrum */
    int32_t target_on_device;   /* 1: target is a device pointer */
    int32_t checkpoint_every;   /* accepted steps between stored states, 1..16 (0: 16) */
    double camera_delta;        /* central-difference step of the camera
                                   transform in a and inclination (0: 1e-6) */
    double* per_ray_grad;       /* NULL, or host [P][5]: each ray's share of grad */
    int32_t escape_rays;        /* rays that take a polar escape (pass within about
                                   1e-8 rad of the axis): 0 differentiate through the
                                   escape (spike guard, escape_cuts); 1 leave them out
                                   of the gradient (their loss still counts). Their
                                   discrete loss is not smooth at finite-difference
                                   scales, and the FP32-stage path reaches the axis
                                   differently from the FP64 one. */
    int32_t reserved;
    /* ray subset (for sharding one image over GPUs): pixels ray_begin + k *
       ray_stride, k < ray_count; ray_count 0: to the end, ray_stride 0: 1.
       The loss and gradient are the subset's; out receives its pixels (the
       others are zero). */
    int64_t ray_begin;
    int64_t ray_count;
    int64_t ray_stride;
} rtw_adjoint_params;

typedef struct rtw_adjoint_result {
    double loss;
    double grad[RTW_ADJOINT_PARAMS];  /* dL/d(a, inclination, n_e0, b_0, theta_e0) */
    double forward_ms;          /* recording forward pass (image, step sizes, checkpoints) */
    double record_ms;           /* between the first recording pass and the reverse sweep: the
                                   pass of rays that outgrew their region, the host scan and
                                   queue order, and the second recording pass of the rays with
                                   a polar escape whose gradient is wanted (state before every
                                   event) */
    double reverse_ms;          /* reverse sweep */
    double total_ms;            /* the whole call, device time */
    uint64_t events;            /* recorded steps: accepted DP45 steps + polar escapes */
    uint64_t checkpoints;       /* stored states */
    uint64_t scratch_bytes;     /* device memory of the records and the sweep */
    uint64_t escape_rays;       /* rays with at least one polar escape */
    uint64_t escape_cuts;       /* polar escapes whose local derivative was a spike
                                   (cotangent growth > 1e3) and that were carried as
                                   the identity instead */
} rtw_adjoint_result;

/* Forward render of one camera of a RTW_SCENE_KERR_SYNCHRO_TORUS scene, the
 * loss against params->target and its gradient. out (may be NULL) receives
 * the forward outputs (spectrum, class, steps) like rtw_render. */
rtw_status rtw_adjoint(rtw_ctx* ctx, const rtw_scene* scene, const rtw_camera* cam,
                       const rtw_render_params* params, const rtw_adjoint_params* adj,
                       rtw_outputs* out, rtw_adjoint_result* result);

/* Host FP64 evaluation of the torus right-hand side in the reference's state
 * layout (state[8 + 2N] = x^mu, k^mu, then (I_c, tau_c) per bin), with the
 * forward kernel's functions (form 0) or the adjoint's generic ones (form 1:
 * geodesic acceleration from metric derivatives). For tests. */
rtw_status rtw_torus_rhs(const rtw_scene* scene, const double* colors_nm, int32_t n_colors, int32_t form,
                         const double* state, double* slope);

/* Host FP64 vector-Jacobian product of the torus right-hand side, the
 * adjoint kernel's own function: mu = J^T cot (reference layout) and
 * pbar[5] = (d slope / d(a, -, n_e0, b_0, theta_e0))^T cot (pbar[1] = 0). */
rtw_status rtw_torus_vjp(const rtw_scene* scene, const double* colors_nm, int32_t n_colors,
                         const double* state, const double* cot, double* mu, double* pbar);

/* Host evaluation of the wormhole skybox's cube-map neighbour rule (cube_wrap,
 * gen_geometry.jl:128-344), the one the ray-bundle lookup uses: texel (i, j)
 * of face `face` (1-based, n texels per face edge) moved by x along i and y
 * along j; out[3] = (i, j, face) after the move. For tests. */
rtw_status rtw_skybox_wrap(int32_t i, int32_t j, int32_t face, int32_t x, int32_t y, int32_t n, int32_t* out);

/* Host FP64 reverse of one FSAL Dormand-Prince step of size h from state of
 * the torus (reference layout): mu = the cotangent of the start state given
 * cot for the end state, pbar the parameter part, hbar = d loss / d h; form 0
 * is the adjoint kernel's structured reverse, form 1 the generic one over the
 * whole state, form 2 the structured one with the optical depths run back
 * from the end of the step (the adjoint kernel's form), form 3 form 2 with
 * FP32 bin partials (the FP32-mixed adjoint's). For tests. */
rtw_status rtw_torus_step_vjp(const rtw_scene* scene, const double* colors_nm, int32_t n_colors,
                              const double* state, double h, const double* cot, int32_t form, double* mu,
                              double* pbar, double* hbar);

/* Host FP64 polar escape of the torus (n_sub sub-steps z <- keep(z - temp
 * f(z)), temp from the state; Kerr source_geometry.jl:249-269 with
 * integrators_LttM.jl:62-105) and the adjoint kernel's vector-Jacobian product
 * of it: end_state, mu = J^T cot, pbar as rtw_torus_vjp. Returns RTW_ERR_NAN
 * when the adjoint's spike guard replaced the escape's derivative by the
 * identity. For tests. */
rtw_status rtw_torus_escape_vjp(const rtw_scene* scene, const double* colors_nm, int32_t n_colors,
                                const double* state, int32_t n_sub, const double* cot, double* end_state,
                                double* mu, double* pbar);

/* Measured issue peaks of this GPU from short in-library microbenchmarks:
 * FP32 FMA, FP64 FMA (flop/s, an FMA counted as 2) and MUFU ex2 (op/s). */
rtw_status rtw_measure_peaks(rtw_ctx* ctx, double* fp32_flops, double* fp64_flops,
                             double* mufu_ops);

/* Evaluates a scene's right-hand side on the host with the trace kernel's own
 * device functors, in FP64 (fp32 = 0) or in the FP32 form of the mixed path
 * (fp32 = 1; host sin/cos/exp stand in for the device's MUFU forms). The
 * geodesic and common-tau part of calc_ray_derivative!
 * (integrators_LttM.jl:9-48): state[9] = (t, r, theta, phi, k^t, k^r,
 * k^theta, k^phi, tau) -> slope[9]; emit[3] (may be NULL) = the emitter
 * numbers A = a_nu emission_scale exp(-tau) / g, X = f_factor g / T and
 * ktau = -a_nu / g, from which the intensity slope of bin c is
 * -A / (exp(X nu_c) - 1). */
rtw_status rtw_scene_rhs(const rtw_scene* scene, int32_t fp32, const double* state, double* slope, double* emit);

/* The reference's gaunt_ei_therm_van_Hoof (emission_functions.jl:54-78) as
 * the bremsstrahlung kernels evaluate it: the Gaunt factor at gam2 and u from
 * the table lut (layout of rtw_render_params.gaunt_lut), in Float32 with the
 * reference's index offsets and its 1.2 outside the table. For tests. */
float rtw_gaunt_lookup(const float* lut, double gam2, double u);

/* Right-hand side of a RTW_SCENE_KERR_BREMS_TORUS scene on the host with the
 * kernels' own functions in FP64 (the layout of rtw_torus_rhs: state[8 + 2N]
 * = (x^mu, k^mu, I_1, tau_1, ..., I_N, tau_N)), with the Gaunt table gaunt_lut
 * (layout of rtw_render_params.gaunt_lut). For tests. */
rtw_status rtw_brems_rhs(const rtw_scene* scene, const double* colors_nm, int32_t n_colors,
                         const float* gaunt_lut, const double* state, double* slope);

/* Limits of rtw_render_noalloc. */
#define RTW_NOALLOC_MAX_FRAMES 64
#define RTW_NOALLOC_SCRATCH_BYTES (24u << 20)

/* Renders like rtw_render but allocates nothing, for callers that cannot call
 * cudaMalloc (a host that owns all device memory up front, a real-time loop
 * that must not enter the allocator) or that hold no rtw_ctx. No counterpart
 * in the reference. Scratch, frame table, bin table and work counter are
 * file-scope __device__ arrays of the library (24 MiB of scratch; every GPU
 * that loads the library holds them until exit). Outputs must be device
 * pointers; at most RTW_NOALLOC_MAX_FRAMES cameras; the scratch caps the
 * resident warps, so it runs slower than rtw_render. Larger requests return
 * RTW_ERR_INVALID_PARAM (text in rtw_noalloc_last_error). Runs on the current
 * device and on params->stream (NULL: default stream, returns when done).
 * block_warps, ctas_per_sm and refill_min are honoured as rtw_render takes
 * them; graph, autotune and trace_ray >= 0 need a context and return
 * RTW_ERR_UNSUPPORTED. The frame and bin tables travel as kernel parameters,
 * so the call reads no host memory after it returns.
 * Calls share the arrays: calls that overlap on the GPU race; serialise them.
 * The first call on a device looks up the arrays' addresses
 * (cudaGetSymbolAddress) and caches them; make it before any stream capture.
 * The cache does not survive cudaDeviceReset: do not call this entry point
 * again in a process after a reset of its device. */
rtw_status rtw_render_noalloc(const rtw_scene* scene, const rtw_camera* cams, int32_t n_cams,
                              const rtw_render_params* params, rtw_outputs* out);
/* Text of the calling thread's last rtw_render_noalloc error ("" if none). */
const char* rtw_noalloc_last_error(void);

/* Operation counts used for the roofline of a render (see rtw_op_counts above). */
rtw_status rtw_get_op_counts(int32_t kind, rtw_op_counts* out);

#ifdef __cplusplus
}
#endif

#endif /* RTW_H */
