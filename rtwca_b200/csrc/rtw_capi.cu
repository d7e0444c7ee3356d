// rtw_capi.cu - host side of the C ABI declared in include/rtw.h: context,
// camera set-up (FP64), CIE tables, validation, device buffers, launch.
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "rtw_internal.h"

namespace rtw {
cudaError_t launch_kind_0(const KParams&, int, int, int, cudaStream_t);
cudaError_t launch_kind_1(const KParams&, int, int, int, cudaStream_t);
cudaError_t launch_kind_2(const KParams&, int, int, int, cudaStream_t);
cudaError_t launch_kind_3(const KParams&, int, int, int, cudaStream_t);
const void* kernel_ptr_0(int, int);
const void* kernel_ptr_1(int, int);
const void* kernel_ptr_2(int, int);
const void* kernel_ptr_3(int, int);

static const void* kernel_ptr(int kind, int precision, int np) {
    switch (kind) {
    case 0: return kernel_ptr_0(precision, np);
    case 1: return kernel_ptr_1(precision, np);
    case 2: return kernel_ptr_2(precision, np);
    default: return kernel_ptr_3(precision, np);
    }
}

static cudaError_t launch_one(const KParams& p, int precision, int grid, int block, cudaStream_t stream) {
    switch (p.sc.kind) {
    case 0: return launch_kind_0(p, precision, grid, block, stream);
    case 1: return launch_kind_1(p, precision, grid, block, stream);
    case 2: return launch_kind_2(p, precision, grid, block, stream);
    default: return launch_kind_3(p, precision, grid, block, stream);
    }
}

// The trace kernel; with a tail queue (FP32-mixed), the main pass and then,
// on the same stream, the tail pass over the rays the main pass queued.
cudaError_t launch_trace(const KParams& p, int precision, int grid, int block, cudaStream_t stream) {
    const cudaError_t e = launch_one(p, precision, grid, block, stream);
    if (e != cudaSuccess || !p.tail || precision != RTW_PREC_MIXED) return e;
    KParams q = p;
    q.tail_mode = 1;
    return launch_one(q, precision, grid, block, stream);
}

size_t spec_bytes_per_warp(int precision, int np) {
    return precision == RTW_PREC_MIXED ? (size_t)3 * 32 * np * sizeof(float) : (size_t)2 * 32 * np * sizeof(double);
}

size_t trace_dyn_smem(int precision, int np, int warps) {
#if RTW_SPEC_SHARED
    if (precision == RTW_PREC_MIXED && np <= 64) return (size_t)warps * 2 * 32 * np * sizeof(float);
#endif
    return 0;
}

cudaError_t trace_allow_smem(int kind, int precision, int np) {
    const size_t bytes = trace_dyn_smem(precision, np, 4);  // the largest CTA: 4 warps
    if (!bytes) return cudaSuccess;
    const void* fn = kernel_ptr(kind, precision, np);
    cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    if (e != cudaSuccess) return e;
    return cudaFuncSetAttribute(fn, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
}

cudaError_t trace_attributes(int kind, int precision, int np, cudaFuncAttributes* attr) {
    return cudaFuncGetAttributes(attr, kernel_ptr(kind, precision, np));
}

namespace {

constexpr double kPi = 3.141592653589793;
constexpr double kNoDivZero = 1e-24;
constexpr double kLightC = 299792458.0;

typedef double M4[4][4];

void mul4(const M4 a, const M4 b, M4 c) {
    M4 t;
    for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 4; ++j) {
            double s = 0;
            for (int k = 0; k < 4; ++k) s += a[i][k] * b[k][j];
            t[i][j] = s;
        }
    std::memcpy(c, t, sizeof(M4));
}

// roll-pitch-yaw R_z R_y R_x (gen_geometry.jl:9-40)
void rot_intrinsic(const double* p, M4 out) {
    M4 rx = {{0}}, ry = {{0}}, rz = {{0}}, t;
    const double c0 = std::cos(p[0]), s0 = std::sin(p[0]);
    const double c1 = std::cos(p[1]), s1 = std::sin(p[1]);
    const double c2 = std::cos(p[2]), s2 = std::sin(p[2]);
    rx[0][0] = 1; rx[1][1] = 1; rx[2][2] = c0; rx[3][2] = s0; rx[2][3] = -s0; rx[3][3] = c0;
    ry[0][0] = 1; ry[1][1] = c1; ry[3][1] = -s1; ry[2][2] = 1; ry[1][3] = s1; ry[3][3] = c1;
    rz[0][0] = 1; rz[1][1] = c2; rz[2][1] = s2; rz[1][2] = -s2; rz[2][2] = c2; rz[3][3] = 1;
    mul4(rz, ry, t);
    mul4(t, rx, out);
}

// rotation of the tetrad axes onto the velocity direction, Rodrigues form,
// transposed, then the yaw fix pi/2 + direction[2] (gen_geometry.jl:47-87)
void rot_final(const double* dir, M4 out) {
    const double d0 = std::sin(dir[0]) * std::cos(dir[1]);
    const double d1 = std::sin(dir[0]) * std::sin(dir[1]);
    double kx = -d1, ky = d0, kz = 0.0;  // (0,0,1) x d
    const double mag = std::sqrt(kx * kx + ky * ky + kz * kz);
    const double yaw[3] = {0, 0, kPi / 2 + dir[1]};
    M4 ry;
    rot_intrinsic(yaw, ry);
    if (!(mag > 0)) {
        std::memcpy(out, ry, sizeof(M4));
        return;
    }
    kx /= mag; ky /= mag; kz /= mag;
    const double K[3][3] = {{0, -kz, ky}, {kz, 0, -kx}, {-ky, kx, 0}};
    const double sa = std::sin(dir[0]), ca = 1 - std::cos(dir[0]);
    M4 r4 = {{0}};
    r4[0][0] = 1;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            double kk = 0;
            for (int m = 0; m < 3; ++m) kk += K[i][m] * K[m][j];
            // stored transposed
            r4[1 + j][1 + i] = (i == j ? 1.0 : 0.0) + sa * K[i][j] + ca * kk;
        }
    mul4(r4, ry, out);
}

// z boost (gen_geometry.jl:93-103)
void boost(double beta, M4 out) {
    std::memset(out, 0, sizeof(M4));
    const double g = 1 / std::sqrt(1 - beta * beta);
    out[0][0] = g; out[3][0] = -beta * g; out[0][3] = -beta * g;
    out[1][1] = 1; out[2][2] = 1; out[3][3] = g;
}

bool is_kerr(int kind) {
    return kind == RTW_SCENE_KERR_DISK || kind == RTW_SCENE_KERR_THICK_DISK || kind == RTW_SCENE_KERR_SYNCHRO_TORUS ||
           kind == RTW_SCENE_KERR_POWEHI || kind == RTW_SCENE_KERR_BREMS_TORUS;
}

double horizon_radius(const rtw_scene& s) {
    if (is_kerr(s.kind)) return s.mass + std::sqrt(s.mass * s.mass - s.spin * s.spin);
    if (s.kind == RTW_SCENE_SCHWARZSCHILD_DISK) return 2 * s.mass;
    return 0.0;
}

// Wormhole.source r(l) (source_geometry.jl:7-31) for the camera's tetrad
double wormhole_r_host(const rtw_scene& s, double l) {
    const double c = kPi / (2 * std::sqrt(2.0));
    const double w_over_m = -std::log(1 / std::cos(c)) + c * std::tan(c);
    const double M = s.edge_out / w_over_m;
    if (!(std::fabs(l) > s.edge_in)) return s.r_in;
    const double x = 2 * (std::fabs(l) - s.edge_in) / (kPi * M);
    return s.r_in + M * (x * std::atan(x) - std::log(1 + x * x) / 2);
}

// inverse tetrad at the camera (calc_inv_vierbein of each scene)
void inv_tetrad(const rtw_scene& s, const double* x, M4 e) {
    for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 4; ++j) e[i][j] = i == j ? 1.0 : 0.0;
    if (s.kind == RTW_SCENE_SYNCHRO_TEST || s.kind == RTW_SCENE_MINKOWSKI_CART_SPHERE)
        return;  // Cartesian Minkowski: the identity
    if (s.kind == RTW_SCENE_WORMHOLE) {            // Wormhole.source/source_geometry.jl:83-90
        const double rl = wormhole_r_host(s, x[1]);
        e[2][2] = 1 / rl;
        e[3][3] = 1 / (rl * std::sin(x[2]) + kNoDivZero);
        return;
    }
    const double r = x[1], th = x[2];
    if (is_kerr(s.kind)) {
        const double a = s.spin, rs = 2 * s.mass;
        const double sig = r * r + (a * std::cos(th)) * (a * std::cos(th));
        const double del = r * r - r * rs + a * a;
        const double A = (r * r + a * a) * sig + rs * r * (a * std::sin(th)) * (a * std::sin(th));
        e[0][0] = std::sqrt(A / (sig * del));
        e[3][0] = (rs * a * r / A) * e[0][0];
        e[1][1] = std::sqrt(del / sig);
        e[2][2] = 1 / std::sqrt(sig);
        e[3][3] = std::sqrt(sig / A) / std::sin(th);
    } else if (s.kind == RTW_SCENE_SCHWARZSCHILD_DISK) {
        const double rs = 2 * s.mass;
        e[0][0] = 1 / std::sqrt(1 - rs / r);
        e[1][1] = std::sqrt(1 - rs / r);
        e[2][2] = 1 / r;
        e[3][3] = 1 / (r * std::sin(th) + kNoDivZero);
    } else {
        e[2][2] = 1 / (r + kNoDivZero);
        e[3][3] = 1 / (r * std::sin(th) + kNoDivZero);
    }
}

bool on_singularity(const double* pos) {
    return std::fabs(pos[1]) <= (double)1e-32f || std::fabs(pos[2]) <= (double)1e-32f || std::fabs(pos[2] - kPi) <= 1e-32;
}

// Bardeen-Press-Teukolsky ISCO with the exponents of Kerr.source/source_geometry.jl:20-37
double reference_isco(double M, double a) {
    const double chi = a / M;
    const double z1 = 1 + std::cbrt(1 - chi * chi) * (std::pow(1 + chi, 1.5) + std::pow(1 - chi, 1.5));
    const double z2 = std::sqrt(3 * chi * chi + z1 * z1);
    return (double)(float)(M * (3 + z2 - std::sqrt((3 - z1) * (3 + z1 + 2 * z2))));
}

const double kCie[4][7] = {
    {0.362, 1.056, -0.065, 0.821, 0.286, 1.217, 0.681},
    {442.0, 599.8, 501.1, 568.8, 530.9, 437.0, 459.0},
    {0.0624, 0.0264, 0.0490, 0.0213, 0.0613, 0.0845, 0.0385},
    {0.0374, 0.0323, 0.0382, 0.0247, 0.0322, 0.0278, 0.0725}};

// multi-lobe Gaussian CIE fit (color_theory.jl:11-61)
double cie_fit(double wl, int first, int count) {
    double v = 0;
    for (int i = first; i < first + count; ++i) {
        const double d = wl - kCie[1][i];
        const double inv_w = d >= 0 ? kCie[3][i] : kCie[2][i];
        v += kCie[0][i] * std::exp(-0.5 * (d * inv_w) * (d * inv_w));
    }
    return v;
}

}  // namespace

void make_dev_scene(const rtw_scene& scene, DevScene& d) {
    std::memset(&d, 0, sizeof(d));
    d.kind = scene.kind;
    d.refprec = 0;
    d.M = scene.mass;
    d.a = is_kerr(scene.kind) ? scene.spin : 0.0;
    d.rs = 2 * scene.mass;
    d.r_ev = horizon_radius(scene);
    d.r_in = scene.r_in; d.r_out = scene.r_out;
    d.th_lo = scene.theta_lo; d.th_hi = scene.theta_hi;
    d.T = scene.temperature; d.anu = scene.a_nu;
    d.esc = scene.escape_radius; d.wind = scene.winding_limit;
    d.rho_r0 = scene.rho_r0; d.rho_h = scene.rho_h; d.rho_idx = scene.rho_index; d.t_idx = scene.t_index;
    d.sqrtM = std::sqrt(scene.mass);
    d.r_pm = is_kerr(scene.kind) ? 2 * std::sqrt(scene.mass * scene.mass - scene.spin * scene.spin) : 0.0;
}

// Spatial blocks of the camera's R2, L and R multiplied, R2[2:4,2:4] *
// L[2:4,2:4] * R[2:4,2:4] (initialization.jl:273-275): what takes a ray
// bundle's axis and direction from the canvas to the observer's frame.
void bundle_basis(const rtw_camera& cam, double m3[9]) {
    M4 R, L, R2;
    rot_intrinsic(cam.pointing, R);
    boost(-cam.speed, L);
    rot_final(cam.direction, R2);
    double t[3][3];
    for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) {
            t[a][b] = 0;
            for (int c = 0; c < 3; ++c) t[a][b] += R2[1 + a][1 + c] * L[1 + c][1 + b];
        }
    for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) {
            double v = 0;
            for (int c = 0; c < 3; ++c) v += t[a][c] * R[1 + c][1 + b];
            m3[3 * a + b] = v;
        }
}

}  // namespace rtw

using namespace rtw;

#include "rtw_ctx.h"



extern "C" {

int32_t rtw_abi_version(void) { return RTW_ABI_VERSION; }

rtw_status rtw_create(rtw_ctx** out, int32_t device) {
    if (!out) return RTW_ERR_INVALID_PARAM;
    *out = nullptr;
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n <= 0) return RTW_ERR_NO_DEVICE;
    if (device < 0 || device >= n) return RTW_ERR_INVALID_PARAM;
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) return RTW_ERR_NO_DEVICE;
    if (prop.major != 10) return RTW_ERR_NO_DEVICE;  // built for sm_100a only
    if (cudaSetDevice(device) != cudaSuccess) return RTW_ERR_CUDA;
    rtw_ctx* ctx = new rtw_ctx();
    ctx->device = device;
    ctx->num_sms = prop.multiProcessorCount;
    if (cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess) {
        delete ctx;
        return RTW_ERR_CUDA;
    }
    for (auto& e : ctx->ev) cudaEventCreate(&e);
    if (cudaMalloc((void**)&ctx->d_ctl, 256) != cudaSuccess || cudaMalloc((void**)&ctx->d_bins, 4 * RTW_MAX_BINS * sizeof(double)) != cudaSuccess) {
        rtw_destroy(ctx);
        return RTW_ERR_OOM;
    }
    *out = ctx;
    return RTW_OK;
}

void rtw_destroy(rtw_ctx* ctx) {
    if (!ctx) return;
    cudaSetDevice(ctx->device);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    cudaFree(ctx->d_frames);
    cudaFree(ctx->d_bins);
    cudaFree(ctx->d_ctl);
    cudaFree(ctx->d_spec);
    cudaFree(ctx->d_tail);
    cudaFree(ctx->d_out);
    cudaFree(ctx->d_sink);
    cudaFree(ctx->d_fclock);
    torus_free(ctx->torus);
    if (ctx->gexec) cudaGraphExecDestroy(ctx->gexec);
    if (ctx->h_stage) cudaFreeHost(ctx->h_stage);
    for (auto& e : ctx->ev)
        if (e) cudaEventDestroy(e);
    if (ctx->stream) cudaStreamDestroy(ctx->stream);
    delete ctx;
}

const char* rtw_last_error(const rtw_ctx* ctx) { return ctx ? ctx->err.c_str() : "null context"; }

rtw_status rtw_scene_default(int32_t kind, rtw_scene* s) {
    if (!s) return RTW_ERR_INVALID_PARAM;
    std::memset(s, 0, sizeof(*s));
    s->kind = kind;
    s->mass = 1.0;
    s->escape_radius = 100.0;
    s->winding_limit = 8 * kPi;
    s->rho_r0 = 6.0;
    s->rho_h = 0.1;
    s->rho_index = -2.0;
    s->t_index = -0.75;
    s->theta_lo = 0;
    s->theta_hi = kPi;
    switch (kind) {
    case RTW_SCENE_MINKOWSKI_SPHERE:  // Minkowski_Sphere_Spherical.source/source_model.jl:44-83
        s->r_in = 0; s->r_out = 1; s->temperature = 5778; s->a_nu = 1;
        break;
    case RTW_SCENE_SCHWARZSCHILD_DISK:  // Schwarzschild ... source_model.jl:44-80
        s->r_in = 6; s->r_out = 12; s->theta_lo = 15 * kPi / 32; s->theta_hi = 17 * kPi / 32;
        s->temperature = 5778; s->a_nu = 1;
        break;
    case RTW_SCENE_KERR_DISK:  // Kerr.source: source_geometry.jl:13, source_model.jl:44-80
        s->spin = (double)0.998f;
        s->r_in = reference_isco(1.0, s->spin); s->r_out = 12;
        s->theta_lo = 31 * kPi / 64; s->theta_hi = 33 * kPi / 64;
        s->temperature = 5778; s->a_nu = (double)1e-1f;
        break;
    case RTW_SCENE_KERR_THICK_DISK:
        s->spin = 0.9;
        s->r_in = 2.320883041761887;  // prograde ISCO of a = 0.9
        s->r_out = 30; s->temperature = 1e4; s->a_nu = 0.05;
        break;
    case RTW_SCENE_KERR_SYNCHRO_TORUS:
        // no reference counterpart: n_e = 1e5 (r/6)^-1.5 exp(-z^2/2(0.3 r)^2),
        // B = 10 (r/6)^-1 G, Theta_e = 10 (r/6)^-1, M87* length scale
        // (the map_scale of Powehi.source/source_model.jl:7)
        s->spin = 0.94;
        s->r_in = 6; s->r_out = 40; s->edge_in = 0.5; s->edge_out = 5;
        s->rho_h = 0.3; s->rho_index = -1.5; s->t_index = -1.0; s->b_index = -1.0;
        s->n_e0 = 1e5; s->b_0 = 10; s->theta_e0 = 10; s->length_cm = 9.62e14;
        s->escape_radius = 110;
        break;
    case RTW_SCENE_KERR_BREMS_TORUS:
        // no reference counterpart: the synchrotron torus's fluid (n_e, Theta_e,
        // tapers) radiating thermal bremsstrahlung, denser (n_e0 = 1e8 cm^-3)
        s->spin = 0.94;
        s->r_in = 6; s->r_out = 40; s->edge_in = 0.5; s->edge_out = 5;
        s->rho_h = 0.3; s->rho_index = -1.5; s->t_index = -1.0; s->b_index = -1.0;
        s->n_e0 = 1e8; s->b_0 = 0; s->theta_e0 = 10; s->length_cm = 9.62e14;
        s->escape_radius = 110;
        break;
    case RTW_SCENE_KERR_POWEHI:
        // Powehi.source (the reference's M87* model): a = 0.9 (source_geometry.jl:12),
        // wedge disk r_ISCO..12, 31pi/64..33pi/64, a_nu = 1e-2, T = 5778
        // (source_model.jl:186-190, 229-232); jet n_e0 = 1e7 m^-3, global field
        // B^phi = 10 G (source_model.jl:13, 47-55); map_scale 9.62e12 m (:7)
        s->spin = (double)0.9f;
        s->r_in = reference_isco(1.0, s->spin); s->r_out = 12;
        s->theta_lo = 31 * kPi / 64; s->theta_hi = 33 * kPi / 64;
        s->temperature = 5778; s->a_nu = (double)1e-2f;
        s->n_e0 = 1e7; s->b_0 = 10; s->length_cm = 9.62e14;
        break;
    case RTW_SCENE_SYNCHRO_TEST:
        // Synchro_Test.source: cylinder of radius 1 (source_model.jl:229-236),
        // B^z = 10 G (:47-54), n_e0 = 1e7 m^-3 and map_scale 9.62e12 m
        // (:7-15), rays end at |x| > 100 (:258-275)
        s->r_out = 1; s->n_e0 = 1e7; s->b_0 = 10; s->length_cm = 9.62e14;
        s->escape_radius = 100;
        break;
    case RTW_SCENE_WORMHOLE:
        // Interstellar's Dneg wormhole (Wormhole.source/source_geometry.jl:7-15):
        // rho = 1, a = 0.005 rho, W = 0.05 rho; escape at r(l) > 100, phi > 8 pi
        s->r_in = 1; s->edge_in = 0.005; s->edge_out = 0.05; s->escape_radius = 100;
        break;
    case RTW_SCENE_MINKOWSKI_CART_SPHERE:
        // Minkowski_Sphere_Cartesian.source: sphere of radius 1 (is_fire
        // :82-90), T = 5.778f3 K (:51-55), a_nu = 1f0 / map_scale (:66-77),
        // rays end at |x| > 100 (:158-172)
        s->r_out = 1; s->temperature = 5778; s->a_nu = 1; s->escape_radius = 100;
        break;
    default:
        return RTW_ERR_INVALID_PARAM;
    }
    return RTW_OK;
}

rtw_status rtw_camera_pixels(rtw_camera* cam, int64_t* n_pix) {
    if (!cam || cam->x_pix <= 0 || !(cam->fov_hor > 0 && cam->fov_hor < 180) || !(cam->fov_vert > 0 && cam->fov_vert < 180))
        return RTW_ERR_INVALID_PARAM;
    const double W = std::tan(kPi * cam->fov_hor / 180 / 2), H = std::tan(kPi * cam->fov_vert / 180 / 2);
    const double yp = std::nearbyint(cam->x_pix * H / W);
    if (!(yp >= 1 && yp < 1e9)) return RTW_ERR_INVALID_PARAM;
    cam->y_pix = (int32_t)yp;
    if (n_pix) {
        const bool win = cam->win_w || cam->win_h || cam->win_x0 || cam->win_y0;
        *n_pix = win ? (int64_t)cam->win_w * cam->win_h : (int64_t)cam->x_pix * cam->y_pix;
    }
    return RTW_OK;
}

static rtw_status build_frame(const rtw_scene& s, rtw_camera& cam, FrameDesc& f) {
    rtw_status st = rtw_camera_pixels(&cam, nullptr);
    if (st != RTW_OK) return st;
    // (the Cartesian scenes have no coordinate singularity: Synchro_Test.source/
    // source_geometry.jl:84-88, Minkowski_Sphere_Cartesian.source/source_geometry.jl:80-82)
    if (s.kind == RTW_SCENE_WORMHOLE) {  // the poles only (Wormhole.source/source_geometry.jl:197-205)
        if (std::fabs(cam.position[2]) <= (double)1e-32f || std::fabs(cam.position[2] - kPi) <= (double)1e-32f)
            return RTW_ERR_INVALID_CAMERA;
    } else if (s.kind != RTW_SCENE_SYNCHRO_TEST && s.kind != RTW_SCENE_MINKOWSKI_CART_SPHERE &&
               on_singularity(cam.position)) {
        return RTW_ERR_INVALID_CAMERA;
    }
    if (!(std::fabs(cam.speed) < 1)) return RTW_ERR_INVALID_PARAM;
    const double fh = kPi * cam.fov_hor / 180, fv = kPi * cam.fov_vert / 180;
    f.W = std::tan(fh / 2);
    f.H = std::tan(fv / 2);
    f.rh = 2 * f.W / (cam.x_pix + 1);
    f.rv = 2 * f.H / (cam.y_pix + 1);
    if (cam.win_w == 0 && cam.win_h == 0 && cam.win_x0 == 0 && cam.win_y0 == 0) {
        f.xp = cam.x_pix;
        f.yp = cam.y_pix;
        f.i0 = f.j0 = 0;
    } else {
        if (cam.win_x0 < 0 || cam.win_y0 < 0 || cam.win_w < 1 || cam.win_h < 1 ||
            (int64_t)cam.win_x0 + cam.win_w > cam.x_pix || (int64_t)cam.win_y0 + cam.win_h > cam.y_pix)
            return RTW_ERR_INVALID_PARAM;
        f.xp = cam.win_w;
        f.yp = cam.win_h;
        f.i0 = cam.win_x0;
        f.j0 = cam.win_y0;
    }
    M4 R, L, R2, e, t1, t2, M;
    rot_intrinsic(cam.pointing, R);
    boost(-cam.speed, L);
    rot_final(cam.direction, R2);
    inv_tetrad(s, cam.position, e);
    mul4(e, R2, t1);
    mul4(t1, L, t2);
    mul4(t2, R, M);
    for (int i = 0; i < 4; ++i) f.pos[i] = cam.position[i];
    for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 4; ++j) {
            f.M[4 * i + j] = M[i][j];
            if (!std::isfinite(M[i][j])) return RTW_ERR_NAN;
        }
    if (!(cam.tolerance > 0 && cam.tolerance < 1) || cam.max_steps <= 0) return RTW_ERR_INVALID_PARAM;
    f.tol = cam.tolerance;
    f.r_term = (1 + 10 * cam.tolerance) * horizon_radius(s);
    f.thick = -std::log(cam.tolerance);
    f.max_steps = cam.max_steps;
    return RTW_OK;
}

// Frame descriptors of a batch (used by the allocation-free entry point).
rtw_status rtw_prepare_frames(const rtw_scene* scene, const rtw_camera* cams, int32_t n_cams, void* frames_out,
                              int64_t* total_out) {
    if (!scene || !cams || !frames_out || n_cams <= 0) return RTW_ERR_INVALID_PARAM;
    FrameDesc* frames = static_cast<FrameDesc*>(frames_out);
    long long total = 0;
    for (int f = 0; f < n_cams; ++f) {
        rtw_camera cam = cams[f];
        const rtw_status s = build_frame(*scene, cam, frames[f]);
        if (s != RTW_OK) return s;
        frames[f].ray_begin = total;
        total += (long long)frames[f].xp * frames[f].yp;
    }
    *total_out = total;
    return RTW_OK;
}

rtw_status rtw_camera_rays(const rtw_scene* scene, const rtw_camera* camin, double* rays, int64_t n_pix) {
    if (!scene || !camin || !rays) return RTW_ERR_INVALID_PARAM;
    rtw_camera cam = *camin;
    FrameDesc f;
    rtw_status st = build_frame(*scene, cam, f);
    if (st != RTW_OK) return st;
    if ((int64_t)f.xp * f.yp != n_pix) return RTW_ERR_INVALID_PARAM;
    for (int j = 0; j < f.yp; ++j)
        for (int i = 0; i < f.xp; ++i) {
            double* S = rays + 8 * ((int64_t)i + (int64_t)f.xp * j);
            const double w = f.rh * ((f.i0 + i + 1) - 0.5) - f.W;
            const double hh = f.rv * ((f.j0 + j + 1) - 0.5) - f.H;
            const double th = std::atan(std::sqrt(w * w + hh * hh));
            double ph;
            if (w > 0) ph = std::atan(hh / w);
            else if (w < 0 && hh >= 0) ph = std::atan(hh / w) + kPi;
            else if (w < 0 && hh < 0) ph = std::atan(hh / w) - kPi;
            else if (w == 0 && hh > 0) ph = kPi / 2;
            else if (w == 0 && hh < 0) ph = -kPi / 2;
            else ph = 0;
            const double v[4] = {1, -std::sin(th) * std::cos(ph), -std::sin(th) * std::sin(ph), -std::cos(th)};
            for (int k = 0; k < 4; ++k) S[k] = f.pos[k];
            for (int r = 0; r < 4; ++r) {
                double acc = 0;
                for (int k = 0; k < 4; ++k) acc += f.M[4 * r + k] * v[k];
                S[4 + r] = acc;
            }
        }
    return RTW_OK;
}

rtw_status rtw_cie_weights(const double* colors, int32_t n, double* wx, double* wy, double* wz, double* fac) {
    if (!colors || n <= 0 || n > RTW_MAX_BINS) return RTW_ERR_INVALID_PARAM;
    for (int i = 0; i < n; ++i)
        if (!(colors[i] > 0)) return RTW_ERR_INVALID_PARAM;
    for (int i = 0; i < n; ++i) {
        double w;
        if (n == 1) w = 1.0;
        else if (i == 0) w = (colors[1] - colors[0]) / 2;
        else if (i == n - 1) w = (colors[n - 1] - colors[n - 2]) / 2;
        else w = (colors[i + 1] - colors[i - 1]) / 2;
        if (wx) wx[i] = cie_fit(colors[i], 0, 3) * w;
        if (wy) wy[i] = cie_fit(colors[i], 3, 2) * w;
        if (wz) wz[i] = cie_fit(colors[i], 5, 2) * w;
        const double nu = 1.0 / colors[i];
        if (fac) fac[i] = nu * nu * nu * kLightC / (colors[i] * colors[i]);
    }
    return RTW_OK;
}

}  // extern "C"

namespace {

// Autotuner: times every candidate (warps per CTA x compaction interval) on
// the first camera at up to 768 pixels wide (about ten rays per resident
// lane) and keeps the fastest per (kind, precision, bins, integrator).
rtw_status autotune(rtw_ctx* ctx, const rtw_scene& scene, const rtw_camera& cam0, const rtw_render_params& prm,
                    int np, std::array<int, 2>& choice) {
    const std::array<int, 4> key = {scene.kind, prm.precision, np, prm.integrator};
    for (const auto& kv : ctx->tuned)
        if (kv.first == key) {
            choice = kv.second;
            return RTW_OK;
        }
    rtw_camera cam = cam0;
    cam.x_pix = std::min(cam.x_pix, 768);
    rtw_render_params q = prm;
    q.autotune = 0;
    q.graph = 0;
    q.stream = nullptr;
    q.trace_ray = -1;
    rtw_outputs none;
    std::memset(&none, 0, sizeof(none));
    none.on_device = 1;
    const int warp_c[2] = {4, 2};
    const int refill_c[3] = {1, 4, 8};
    float best = 0;
    choice = {4, 1};
    for (int pass = 0; pass < 2; ++pass)  // pass 0 warms up the default shape
        for (int w : warp_c)
            for (int r : refill_c) {
                if (pass == 0 && (w != 4 || r != 1)) continue;
                q.block_warps = w;
                q.refill_min = r;
                const rtw_status st = rtw_render(ctx, &scene, &cam, 1, &q, &none);
                if (st != RTW_OK) return st;
                float ms = 0;
                cudaEventElapsedTime(&ms, ctx->ev[1], ctx->ev[2]);
                if (pass == 1 && (best == 0 || ms < best)) {
                    best = ms;
                    choice = {w, r};
                }
            }
    ctx->tuned.push_back({key, choice});
    return RTW_OK;
}

}  // namespace

extern "C" {

rtw_status rtw_render(rtw_ctx* ctx, const rtw_scene* scene, const rtw_camera* cams, int32_t n_cams,
                      const rtw_render_params* prm, rtw_outputs* out) {
    if (!ctx) return RTW_ERR_INVALID_PARAM;
    ctx->err.clear();
    if (!scene || !cams || !prm || !out) return fail(ctx, RTW_ERR_INVALID_PARAM, "null argument");
    if (n_cams <= 0 || n_cams > RTW_MAX_FRAMES) return fail(ctx, RTW_ERR_INVALID_PARAM, "n_cams out of range");
    if (prm->n_colors <= 0 || prm->n_colors > RTW_MAX_BINS || !prm->colors_nm)
        return fail(ctx, RTW_ERR_INVALID_PARAM, "n_colors must be 1..128 with colors_nm set");
    if (prm->ray_bundles && scene->kind != RTW_SCENE_WORMHOLE && scene->kind != RTW_SCENE_MINKOWSKI_CART_SPHERE)
        return fail(ctx, RTW_ERR_UNSUPPORTED, "ray bundles are built for the skybox scenes only");
    if (scene->kind == RTW_SCENE_KERR_SYNCHRO_TORUS || scene->kind == RTW_SCENE_KERR_POWEHI ||
        scene->kind == RTW_SCENE_SYNCHRO_TEST || scene->kind == RTW_SCENE_WORMHOLE ||
        scene->kind == RTW_SCENE_MINKOWSKI_CART_SPHERE || scene->kind == RTW_SCENE_KERR_BREMS_TORUS)
        return torus_render(ctx, scene, cams, n_cams, prm, out);
    if (scene->ref_precision) return fail(ctx, RTW_ERR_UNSUPPORTED, "ref_precision is an oracle-only switch");
    if (prm->precision != RTW_PREC_FP64 && prm->precision != RTW_PREC_MIXED && prm->precision != RTW_PREC_FP64_PLAIN)
        return fail(ctx, RTW_ERR_INVALID_PARAM, "precision");
    const bool plain = prm->precision == RTW_PREC_FP64_PLAIN;
    if (prm->integrator != RTW_DP45_REF_COMPAT && prm->integrator != RTW_DP45_FSAL)
        return fail(ctx, RTW_ERR_INVALID_PARAM, "integrator");
    if (scene->kind < 0 || scene->kind > RTW_SCENE_KERR_THICK_DISK) return fail(ctx, RTW_ERR_INVALID_PARAM, "scene kind");
    if (!(prm->max_dt_scale > 0)) return fail(ctx, RTW_ERR_INVALID_PARAM, "max_dt_scale must be > 0");
    if (is_kerr(scene->kind) && !(std::fabs(scene->spin) < scene->mass))
        return fail(ctx, RTW_ERR_INVALID_PARAM, "Kerr spin must satisfy |a| < M");
    if (!(scene->mass > 0)) return fail(ctx, RTW_ERR_INVALID_PARAM, "mass must be > 0");
    if (cudaSetDevice(ctx->device) != cudaSuccess) return fail(ctx, RTW_ERR_CUDA, "cudaSetDevice");
    cudaStream_t st = prm->stream ? (cudaStream_t)prm->stream : ctx->stream;

    // frames
    std::vector<FrameDesc> frames(n_cams);
    long long total = 0;
    for (int f = 0; f < n_cams; ++f) {
        rtw_camera cam = cams[f];
        rtw_status s = build_frame(*scene, cam, frames[f]);
        if (s == RTW_ERR_INVALID_CAMERA) return fail(ctx, s, "camera " + std::to_string(f) + " is on a coordinate singularity");
        if (s != RTW_OK) return fail(ctx, s, "camera " + std::to_string(f) + " parameters invalid or non-finite");
        frames[f].ray_begin = total;
        total += (long long)frames[f].xp * frames[f].yp;
    }
    // bins
    const int N = prm->n_colors;
    std::vector<double> bins(4 * RTW_MAX_BINS, 0.0);
    std::vector<double> wx(N), wy(N), wz(N), fac(N);
    if (rtw_cie_weights(prm->colors_nm, N, wx.data(), wy.data(), wz.data(), fac.data()) != RTW_OK)
        return fail(ctx, RTW_ERR_INVALID_PARAM, "colors_nm must be positive");
    for (int c = 0; c < N; ++c) {
        bins[c] = 1.0 / prm->colors_nm[c];
        bins[RTW_MAX_BINS + c] = fac[c] * wx[c];
        bins[2 * RTW_MAX_BINS + c] = fac[c] * wy[c];
        bins[3 * RTW_MAX_BINS + c] = fac[c] * wz[c];
    }
    const int np = N <= 32 ? 32 : (N <= 64 ? 64 : 128);

    // launch shape: explicit values, else the autotuner's choice, else defaults
    int warps = prm->block_warps > 0 ? std::min(prm->block_warps, 4) : 0;  // kernel launch bound: 128 threads
    int refill = prm->refill_min > 0 ? std::min(prm->refill_min, 32) : 0;
    if (prm->autotune && !plain && (warps == 0 || refill == 0)) {
        std::array<int, 2> choice;
        const rtw_status ts = autotune(ctx, *scene, cams[0], *prm, np, choice);
        if (ts != RTW_OK) return ts;
        ctx->err.clear();
        if (warps == 0) warps = choice[0];
        if (refill == 0) refill = choice[1];
    }
    if (warps == 0) warps = 4;
    if (refill == 0) refill = 1;
    const int block = 32 * warps;
    if (!plain) RTW_CUDA(trace_allow_smem(scene->kind, prm->precision, np), "kernel shared-memory attribute");
    int per_sm = prm->ctas_per_sm;
    if (per_sm <= 0) {
        int occ = 0;
        RTW_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kernel_ptr(scene->kind, prm->precision, np), block,
                                                               trace_dyn_smem(prm->precision, np, warps)),
                 "occupancy query");
        per_sm = std::max(1, occ);
    }
    const int grid = ctx->num_sms * per_sm;
    const size_t spec_need = (size_t)grid * warps * spec_bytes_per_warp(prm->precision, np);

    rtw_status s;
    if ((s = ensure(ctx, &ctx->d_frames, &ctx->frames_cap, sizeof(FrameDesc) * n_cams)) != RTW_OK) return s;
    if ((s = ensure(ctx, &ctx->d_spec, &ctx->spec_cap, spec_need)) != RTW_OK) return s;
    // the FP32-mixed tail queue: room for a quarter of the rays (at least
    // 65536); rays past it stay in their lanes
    const bool use_tail = prm->precision == RTW_PREC_MIXED && prm->tail_pass >= 0 && !plain;
    long long tail_cap = 0;
    if (use_tail) {
        tail_cap = std::min<long long>(total, std::max<long long>(65536, total / 4));
        const size_t rec = ((sizeof(TailRec) * (size_t)tail_cap + 255) & ~(size_t)255);
        if ((s = ensure(ctx, &ctx->d_tail, &ctx->tail_bytes, rec + sizeof(float) * 3 * np * (size_t)tail_cap)) != RTW_OK)
            return s;
    }
    if ((s = ensure(ctx, (void**)&ctx->d_fclock, &ctx->fclock_cap, sizeof(unsigned long long) * 3 * n_cams)) != RTW_OK)
        return s;

    // outputs
    float* xyz = out->xyz;
    uint8_t* cls = out->term_class;
    uint32_t* steps = out->steps;
    float* spectrum = out->spectrum;
    double* fstate = out->final_state;
    float* tau = out->tau;
    double* trace = out->trace;
    const bool tracing = prm->trace_ray >= 0 && out->trace && out->trace_capacity > 0;
    size_t off_xyz = 0, off_cls = 0, off_steps = 0, off_spec = 0, off_state = 0, off_tau = 0, off_trace = 0;
    if (!out->on_device) {
        size_t o = 0;
        auto take = [&](bool want, size_t bytes, size_t& off) {
            if (want) {
                off = o;
                o += (bytes + 255) & ~(size_t)255;
            }
        };
        take(xyz != nullptr, sizeof(float) * 3 * total, off_xyz);
        take(cls != nullptr, sizeof(uint8_t) * total, off_cls);
        take(steps != nullptr, sizeof(uint32_t) * total, off_steps);
        take(spectrum != nullptr, sizeof(float) * N * total, off_spec);
        take(fstate != nullptr, sizeof(double) * 8 * total, off_state);
        take(tau != nullptr, sizeof(float) * total, off_tau);
        take(tracing, sizeof(double) * RTW_TRACE_FIELDS * (size_t)out->trace_capacity, off_trace);
        if ((s = ensure(ctx, &ctx->d_out, &ctx->out_cap, std::max<size_t>(o, 256))) != RTW_OK) return s;
        char* base = (char*)ctx->d_out;
        xyz = xyz ? (float*)(base + off_xyz) : nullptr;
        cls = cls ? (uint8_t*)(base + off_cls) : nullptr;
        steps = steps ? (uint32_t*)(base + off_steps) : nullptr;
        spectrum = spectrum ? (float*)(base + off_spec) : nullptr;
        fstate = fstate ? (double*)(base + off_state) : nullptr;
        tau = tau ? (float*)(base + off_tau) : nullptr;
        trace = tracing ? (double*)(base + off_trace) : nullptr;
    }

    KParams p;
    std::memset(&p, 0, sizeof(p));
    make_dev_scene(*scene, p.sc);
    p.frames = (const FrameDesc*)ctx->d_frames;
    p.n_frames = n_cams;
    p.n_bins = N;
    p.total_rays = total;
    p.max_dt_scale = prm->max_dt_scale;
    // promotion thresholds: < 0 disables, 0 takes the default. Horizon:
    // r - r+ < 1e-3 M; there the radial acceleration is a sum of O(1/Delta)
    // terms that cancel to O(1) and FP32 stages lose every digit before the
    // (1 + 10 tol) r+ stop. Poles: sin(theta) < 1e-2.
    const double pdr = prm->promote_dr < 0 ? -1.0 : (prm->promote_dr > 0 ? prm->promote_dr : 1e-3);
    // pole promotion of the trace kernel: default sin(theta) < 2e-3 (1e-2 measured
    // 4 % slower on the Kerr disk, with the same parity: near-axis FP64 attempts
    // hold their whole warp)
    const double psn = prm->promote_sin < 0 ? 0.0 : (prm->promote_sin > 0 ? std::min(prm->promote_sin, 1.0) : 2e-3);
    p.promote_dr = pdr * scene->mass;
    p.promote_theta = std::asin(psn);
    p.fsal = prm->integrator == RTW_DP45_FSAL;
    p.pixel_order = prm->pixel_order;
    p.bin_nu = ctx->d_bins;
    p.bin_fx = ctx->d_bins + RTW_MAX_BINS;
    p.bin_fy = ctx->d_bins + 2 * RTW_MAX_BINS;
    p.bin_fz = ctx->d_bins + 3 * RTW_MAX_BINS;
    p.spec = ctx->d_spec;
    p.np = np;
    p.counter = ctx->d_ctl;
    p.stats = (DevStats*)(ctx->d_ctl + 1);
    p.xyz = xyz; p.cls = cls; p.steps = steps; p.spectrum = spectrum; p.final_state = fstate; p.tau = tau;
    p.trace = tracing ? trace : nullptr;
    p.trace_gid = tracing ? prm->trace_ray : -1;
    p.trace_cap = tracing ? out->trace_capacity : 0;
    p.refill_min = refill;
    p.frame_clock = ctx->d_fclock;
    if (use_tail) {
        p.tail = (TailRec*)ctx->d_tail;
        p.tail_spec = (float*)((char*)ctx->d_tail + ((sizeof(TailRec) * (size_t)tail_cap + 255) & ~(size_t)255));
        p.tail_cap = tail_cap;
    }
    ctx->last_tail_cap = use_tail ? tail_cap : 0;

    const size_t frames_bytes = sizeof(FrameDesc) * n_cams;
    const size_t bins_bytes = sizeof(double) * 4 * RTW_MAX_BINS;
    // the launch sequence up to the kernel: frame and bin tables, counter
    // resets, kernel, with events around the kernel
    // (under stream capture the events are recorded as external event nodes,
    // so that every replay records them)
    auto enqueue = [&](const void* src_frames, const void* src_bins, bool capturing) -> cudaError_t {
        auto record = [&](cudaEvent_t ev) {
            return capturing ? cudaEventRecordWithFlags(ev, st, cudaEventRecordExternal) : cudaEventRecord(ev, st);
        };
        cudaError_t e;
        if ((e = record(ctx->ev[0])) != cudaSuccess) return e;
        if ((e = cudaMemcpyAsync(ctx->d_frames, src_frames, frames_bytes, cudaMemcpyHostToDevice, st)) != cudaSuccess) return e;
        if ((e = cudaMemcpyAsync(ctx->d_bins, src_bins, bins_bytes, cudaMemcpyHostToDevice, st)) != cudaSuccess) return e;
        // counters: 1 + 12 words of the 256-byte control block
        if ((e = cudaMemsetAsync(ctx->d_ctl, 0, sizeof(unsigned long long) + sizeof(DevStats), st)) != cudaSuccess) return e;
        if ((e = cudaMemsetAsync(ctx->d_fclock, 0, sizeof(unsigned long long) * 3 * n_cams, st)) != cudaSuccess) return e;
        if (p.trace)  // all-ones bytes: NaN records mark the unused tail
            if ((e = cudaMemsetAsync(p.trace, 0xff, sizeof(double) * RTW_TRACE_FIELDS * (size_t)p.trace_cap, st)) != cudaSuccess)
                return e;
        if ((e = record(ctx->ev[1])) != cudaSuccess) return e;
        if (plain) {
            // one thread per pixel over the whole image, as the reference's grid
            const long long g = std::max<long long>(1, (total + 127) / 128);
            e = launch_plain(p, (int)std::min<long long>(g, 1 << 30), 128, st);
        } else {
            e = launch_trace(p, prm->precision, grid, block, st);
        }
        if (e != cudaSuccess) return e;
        return record(ctx->ev[2]);
    };
    int replayed = 0;
    if (prm->graph) {
        // pinned staging for the tables (a captured copy reads its source
        // address at every replay); wait until the previous render has read it
        if (ctx->have_last) RTW_CUDA(cudaEventSynchronize(ctx->ev[1]), "previous render");
        if (ctx->stage_cap < frames_bytes + bins_bytes) {
            if (ctx->gexec) cudaGraphExecDestroy(ctx->gexec);
            ctx->gexec = nullptr;
            if (ctx->h_stage) cudaFreeHost(ctx->h_stage);
            ctx->h_stage = nullptr;
            ctx->stage_cap = 0;
            RTW_CUDA(cudaHostAlloc(&ctx->h_stage, frames_bytes + bins_bytes, cudaHostAllocDefault), "pinned staging");
            ctx->stage_cap = frames_bytes + bins_bytes;
        }
        char* stage = (char*)ctx->h_stage;
        std::memcpy(stage, frames.data(), frames_bytes);
        std::memcpy(stage + frames_bytes, bins.data(), bins_bytes);
        // replay while everything the capture baked in is unchanged
        std::vector<unsigned char> key(sizeof(KParams) + 4 * sizeof(int) + sizeof(void*));
        unsigned char* k = key.data();
        std::memcpy(k, &p, sizeof(KParams));
        const int shape[4] = {grid, block, prm->precision, n_cams};
        std::memcpy(k + sizeof(KParams), shape, sizeof(shape));
        std::memcpy(k + sizeof(KParams) + sizeof(shape), &st, sizeof(void*));
        if (ctx->gexec && key == ctx->gkey) {
            replayed = 1;
        } else {
            if (ctx->gexec) cudaGraphExecDestroy(ctx->gexec);
            ctx->gexec = nullptr;
            ctx->gkey.clear();
            RTW_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal), "graph capture");
            const cudaError_t eq = enqueue(stage, stage + frames_bytes, true);
            cudaGraph_t g = nullptr;
            const cudaError_t ec = cudaStreamEndCapture(st, &g);
            if (eq != cudaSuccess) {
                if (g) cudaGraphDestroy(g);
                return cuda_fail(ctx, eq, "graph capture of the launch");
            }
            if (ec != cudaSuccess) return cuda_fail(ctx, ec, "graph capture end");
            const cudaError_t ei = cudaGraphInstantiate(&ctx->gexec, g, 0);
            cudaGraphDestroy(g);
            if (ei != cudaSuccess) {
                ctx->gexec = nullptr;
                return cuda_fail(ctx, ei, "graph instantiate");
            }
            ctx->gkey = key;
        }
        RTW_CUDA(cudaGraphLaunch(ctx->gexec, st), "graph launch");
    } else {
        RTW_CUDA(enqueue(frames.data(), bins.data(), false), "trace launch sequence");
    }
    if (!out->on_device) {
        if (out->xyz) RTW_CUDA(cudaMemcpyAsync(out->xyz, xyz, sizeof(float) * 3 * total, cudaMemcpyDeviceToHost, st), "xyz D2H");
        if (out->term_class) RTW_CUDA(cudaMemcpyAsync(out->term_class, cls, total, cudaMemcpyDeviceToHost, st), "class D2H");
        if (out->steps) RTW_CUDA(cudaMemcpyAsync(out->steps, steps, sizeof(uint32_t) * total, cudaMemcpyDeviceToHost, st), "steps D2H");
        if (out->spectrum) RTW_CUDA(cudaMemcpyAsync(out->spectrum, spectrum, sizeof(float) * N * total, cudaMemcpyDeviceToHost, st), "spectrum D2H");
        if (out->final_state) RTW_CUDA(cudaMemcpyAsync(out->final_state, fstate, sizeof(double) * 8 * total, cudaMemcpyDeviceToHost, st), "state D2H");
        if (out->tau) RTW_CUDA(cudaMemcpyAsync(out->tau, tau, sizeof(float) * total, cudaMemcpyDeviceToHost, st), "tau D2H");
        if (tracing)
            RTW_CUDA(cudaMemcpyAsync(out->trace, trace, sizeof(double) * RTW_TRACE_FIELDS * (size_t)out->trace_capacity,
                                     cudaMemcpyDeviceToHost, st), "trace D2H");
    }
    RTW_CUDA(cudaEventRecord(ctx->ev[3], st), "event");
    ctx->have_last = true;
    std::memset(&ctx->last, 0, sizeof(ctx->last));
    ctx->last.rays = (uint64_t)total;
    ctx->last_frames = n_cams;
    ctx->last_grid = grid;
    ctx->last_warps = warps;
    ctx->last_refill = refill;
    ctx->last_replayed = replayed;
    ctx->last_launches = use_tail ? 2 : 1;
    if (!prm->stream) {
        RTW_CUDA(cudaStreamSynchronize(st), "trace kernel");
    }
    return RTW_OK;
}

rtw_status rtw_get_stats(rtw_ctx* ctx, rtw_stats* out) {
    if (!ctx || !out) return RTW_ERR_INVALID_PARAM;
    if (!ctx->have_last) return fail(ctx, RTW_ERR_INVALID_PARAM, "no render yet");
    RTW_CUDA(cudaSetDevice(ctx->device), "cudaSetDevice");
    RTW_CUDA(cudaEventSynchronize(ctx->ev[3]), "sync");
    DevStats ds;
    RTW_CUDA(cudaMemcpy(&ds, ctx->d_ctl + 1, sizeof(ds), cudaMemcpyDeviceToHost), "stats D2H");
    float k = 0, t = 0;
    cudaEventElapsedTime(&k, ctx->ev[1], ctx->ev[2]);
    cudaEventElapsedTime(&t, ctx->ev[0], ctx->ev[3]);
    out->rays = ds.rays;
    out->step_attempts = ds.step_attempts;
    out->rejected_steps = ds.rejected_steps;
    out->promoted_steps = ds.promoted_steps;
    out->spectral_steps = ds.spectral_steps;
    out->emitting_steps = ds.emitting_steps;
    out->escape_substeps = ds.escape_substeps;
    out->nan_rays = ds.nan_rays;
    out->kernel_ms = k;
    out->total_ms = t;
    out->phase_cycles[0] = ds.cyc_refill;
    out->phase_cycles[1] = ds.cyc_geo;
    out->phase_cycles[2] = ds.cyc_spec;
    out->phase_cycles[3] = ds.cyc_commit;
    out->grid = ctx->last_grid;
    out->block_warps = ctx->last_warps;
    out->refill_min = ctx->last_refill;
    out->graph_replayed = ctx->last_replayed;
    out->tail_rays = std::min<unsigned long long>(ds.tail_rays, (unsigned long long)ctx->last_tail_cap);
    out->launches = ctx->last_launches;
    out->reserved0 = 0;
    return RTW_OK;
}

rtw_status rtw_get_frame_times(rtw_ctx* ctx, int32_t n_frames, double* done_ms, double* span_ms) {
    if (!ctx) return RTW_ERR_INVALID_PARAM;
    if (!ctx->have_last || ctx->last_frames <= 0) return fail(ctx, RTW_ERR_INVALID_PARAM, "no render yet");
    if (n_frames != ctx->last_frames) return fail(ctx, RTW_ERR_INVALID_PARAM, "n_frames differs from the last render");
    RTW_CUDA(cudaSetDevice(ctx->device), "cudaSetDevice");
    RTW_CUDA(cudaEventSynchronize(ctx->ev[3]), "sync");
    std::vector<unsigned long long> h((size_t)3 * n_frames);
    RTW_CUDA(cudaMemcpy(h.data(), ctx->d_fclock, sizeof(unsigned long long) * h.size(), cudaMemcpyDeviceToHost),
             "frame clock D2H");
    const unsigned long long* start = h.data() + n_frames;
    const unsigned long long* end = h.data() + 2 * (size_t)n_frames;
    unsigned long long t0 = ~0ull;
    for (int f = 0; f < n_frames; ++f)
        if (start[f]) t0 = std::min(t0, start[f]);
    for (int f = 0; f < n_frames; ++f) {
        const bool ok = start[f] != 0 && end[f] != 0;
        if (done_ms) done_ms[f] = ok ? (double)(end[f] - t0) * 1e-6 : NAN;
        if (span_ms) span_ms[f] = ok ? (double)(end[f] - start[f]) * 1e-6 : NAN;
    }
    return RTW_OK;
}

rtw_status rtw_measure_peaks(rtw_ctx* ctx, double* fp32, double* fp64, double* mufu) {
    if (!ctx) return RTW_ERR_INVALID_PARAM;
    RTW_CUDA(cudaSetDevice(ctx->device), "cudaSetDevice");
    if (!ctx->d_sink) RTW_CUDA(cudaMalloc((void**)&ctx->d_sink, 64), "sink");
    const int block = 256, grid = ctx->num_sms * 8;
    double* outs[3] = {fp32, fp64, mufu};
    const int iters[3] = {4096, 1024, 1024};
    for (int w = 0; w < 3; ++w) {
        // warm-up
        RTW_CUDA(launch_peak_probe(w, grid, block, 16, ctx->d_sink, ctx->stream), "probe");
        RTW_CUDA(cudaEventRecord(ctx->ev[0], ctx->stream), "event");
        RTW_CUDA(launch_peak_probe(w, grid, block, iters[w], ctx->d_sink, ctx->stream), "probe");
        RTW_CUDA(cudaEventRecord(ctx->ev[1], ctx->stream), "event");
        RTW_CUDA(cudaEventSynchronize(ctx->ev[1]), "probe sync");
        float ms = 0;
        cudaEventElapsedTime(&ms, ctx->ev[0], ctx->ev[1]);
        const double ops = (double)grid * block * iters[w] * 16 * 8;
        const double per = (w == 2) ? 1.0 : 2.0;  // FMA = 2 flops
        if (outs[w]) *outs[w] = ops * per / (ms * 1e-3);
    }
    ctx->have_last = false;
    return RTW_OK;
}

}  // extern "C"
