// rtw_plain.cu - the plain FP64 GPU path: the reference's per-pixel algorithm
// as its GPU form lays it out (one thread per pixel over a grid, the whole
// state of 8 + 2N components with one (I, tau) pair per bin, every stage's
// right-hand side evaluating every bin's radiative coefficients), in FP64,
// with none of the trace kernel's reductions (no persistent refill, no
// warp-cooperative bins, no common-tau reduction). It is the baseline the
// trace kernel is measured against (RTW_PREC_FP64_PLAIN).
//
// Follows ray_kernel / integrate_ray (LttM.jl:11-80), calc_ray_derivative!
// (integrators_LttM.jl:9-48) and RKDP_Step_w_buffer! (integrators_LttM.jl:54-224)
// with the scene functors and guards of rtw_scenes.cuh.
#include <cuda_runtime.h>

#include "rtw_trace.cuh"

namespace rtw {

constexpr int kPlainMaxL = 8 + 2 * RTW_MAX_BINS;

// calc_ray_derivative!: geodesic part from the scene functor, then for every
// bin a_nu, j_nu = a_nu B_nu(T) at nu = g nu_c and the two slopes
// -inv(g) j_nu exp(-tau_c) / nu^3 (= ktau emission_scale exp(-tau_c) /
// (exp(X nu_c) - 1) with X = f_factor g / T, ktau = -a_nu / g) and -inv(g) a_nu.
template <class SC>
__device__ void plain_rhs(const KParams& p, const double* R, double* slope) {
    const int N = p.n_bins;
    double z[10], k[9];
    for (int i = 0; i < 8; ++i) z[i] = R[i];
    z[8] = 0;
    z[9] = R[1] - p.sc.r_ev;
    Emit<double> em;
    SC::template rhs<double>(p.sc, z, k, em);
    for (int i = 0; i < 8; ++i) slope[i] = k[i];
    const double ktau = em.ktau;  // -a_nu / g (0 outside the emitter)
    for (int c = 0; c < N; ++c) {
        if (ktau == 0.0) {
            slope[8 + 2 * c] = 0;
            slope[9 + 2 * c] = 0;
            continue;
        }
        const double nu = p.bin_nu[c];
        slope[8 + 2 * c] = ktau * kEmissionScale * exp(-R[9 + 2 * c]) / (exp(em.X * nu) - 1.0);
        slope[9 + 2 * c] = ktau;
    }
}

// calc_terminate (class of the first predicate that holds)
template <int KIND>
__device__ int plain_terminate(const KParams& p, const FrameDesc& f, const double* R, int L) {
    if (R[1] > p.sc.esc) return RTW_CLASS_ESCAPE;
    if (KIND != RTW_SCENE_MINKOWSKI_SPHERE && R[1] <= f.r_term) return RTW_CLASS_HORIZON;
    if (R[3] > p.sc.wind) return RTW_CLASS_WINDING;
    for (int i = 9; i < L; i += 2)
        if (R[i] < f.thick) return 0;
    return RTW_CLASS_THICK;
}

// keepinbounds! on a full state
template <int KIND>
__device__ void plain_keep(double* R) {
    double x[9];
    for (int i = 0; i < 8; ++i) x[i] = R[i];
    x[8] = 0;
    keep_in_bounds<KIND>(x);
    for (int i = 0; i < 8; ++i) R[i] = x[i];
}

template <int KIND>
__global__ void __launch_bounds__(128) plain_kernel(const KParams p) {
    typedef typename SceneOf<KIND>::type SC;
    const int N = p.n_bins, L = 8 + 2 * N;
    double R[kPlainMaxL], k1[kPlainMaxL], ks[6][kPlainMaxL], buf[kPlainMaxL], y[kPlainMaxL];
    unsigned long long c_att = 0, c_rej = 0, c_esc = 0, c_rays = 0, c_nan = 0;
    for (long long id = (long long)blockIdx.x * blockDim.x + threadIdx.x; id < p.total_rays;
         id += (long long)gridDim.x * blockDim.x) {
        ++c_rays;
        int lo = 0, hi = p.n_frames - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (p.frames[mid].ray_begin <= id) lo = mid; else hi = mid - 1;
        }
        const FrameDesc& f = p.frames[lo];
        const long long local = id - f.ray_begin;
        const int pi = (int)(local % f.xp), pj = (int)(local / f.xp);
        double x9[9];
        camera_ray(f, pi, pj, x9);
        for (int i = 0; i < 8; ++i) R[i] = x9[i];
        for (int i = 8; i < L; ++i) R[i] = 0;
        const double tol = f.tol;
        double dt = -pad_max_dt<KIND, double>(p.sc, R, p.max_dt_scale);
        plain_rhs<SC>(p, R, k1);
        bool rejected = false;
        long long steps = 0;
        int cls = 0;
        for (;;) {
            ++c_att;
            const double max_dt = pad_max_dt<KIND, double>(p.sc, R, p.max_dt_scale);
            double temp;
            bool done = false;
            if (near_singularity<KIND>(R, dt, tol, &temp)) {
                for (int i = 0; i < L; ++i) R[i] -= temp * k1[i];
                plain_keep<KIND>(R);
                ++c_esc;
                for (int it = 0; it < 36; ++it) {
                    if (!plain_terminate<KIND>(p, f, R, L)) {
                        plain_rhs<SC>(p, R, k1);
                        for (int i = 0; i < L; ++i) R[i] -= temp * k1[i];
                        plain_keep<KIND>(R);
                        ++c_esc;
                    }
                }
                if (plain_terminate<KIND>(p, f, R, L)) {
                    rejected = false;
                    done = true;
                } else {
                    plain_rhs<SC>(p, R, k1);
                    dt = -pad_max_dt<KIND, double>(p.sc, R, p.max_dt_scale);
                }
            }
            if (!done) {
                const double h = dt;
                // stages 2..7; ks[s - 2] holds k_s
                for (int s = 2; s <= 7; ++s) {
                    for (int i = 0; i < L; ++i) {
                        double acc = init_coef(s - 2) * k1[i];
                        for (int j = 2; j < s; ++j) acc += dp_coef<double>(j - 2, s - 1 - j) * ks[j - 2][i];
                        buf[i] = R[i] + h * acc;
                    }
                    plain_rhs<SC>(p, buf, ks[s - 2]);
                }
                double err = 0;
                for (int i = 0; i < L; ++i) {
                    // 5th-order slope (row 7 of the tableau) and the error estimate
                    const double ns = b1 * k1[i] + b3 * ks[1][i] + b4 * ks[2][i] + b5 * ks[3][i] + b6 * ks[4][i];
                    y[i] = R[i] + h * ns;
                    const double es = e1 * k1[i] + e3 * ks[1][i] + e4 * ks[2][i] + e5 * ks[3][i] + e6 * ks[4][i] +
                                      e7 * ks[5][i];
                    const double d = h * es;
                    const double tl = tol + fmax(fabs(R[i]), fabs(y[i])) * tol;
                    err += (d / tl) * (d / tl);
                    buf[i] = p.fsal ? ks[5][i] : ns;  // the slope carried to the next step
                }
                bool accept;
                double hnext;
                decide<double>(err, L, h, max_dt, rejected, accept, hnext);
                if (accept) {
                    plain_keep<KIND>(y);
                    for (int i = 0; i < L; ++i) {
                        R[i] = y[i];
                        k1[i] = buf[i];
                    }
                    rejected = false;
                } else {
                    plain_keep<KIND>(R);
                    rejected = true;
                    ++c_rej;
                }
                dt = hnext;
            }
            ++steps;
            if (steps >= f.max_steps) cls = RTW_CLASS_MAXSTEPS;
            else cls = plain_terminate<KIND>(p, f, R, L);
            if (cls) break;
        }
        bool fin = true;
        for (int i = 0; i < 8; ++i) fin &= isfinite(R[i]);
        if (!fin) {
            cls = RTW_CLASS_NAN;
            ++c_nan;
        }
        // color: XYZ = sum_c I_c nu_c^3 c / lambda_c^2 W_c (color_theory.jl:67-108)
        const long long og = id;
        double X = 0, Y = 0, Z = 0;
        for (int c = 0; c < N; ++c) {
            const double I = R[8 + 2 * c];
            X += I * p.bin_fx[c];
            Y += I * p.bin_fy[c];
            Z += I * p.bin_fz[c];
            if (p.spectrum) p.spectrum[og * N + c] = (float)I;
        }
        if (p.xyz) {
            p.xyz[3 * og + 0] = (float)X;
            p.xyz[3 * og + 1] = (float)Y;
            p.xyz[3 * og + 2] = (float)Z;
        }
        if (p.cls) p.cls[og] = (uint8_t)cls;
        if (p.steps) p.steps[og] = (uint32_t)steps;
        if (p.final_state)
            for (int i = 0; i < 8; ++i) p.final_state[8 * og + i] = R[i];
        if (p.tau) p.tau[og] = (float)R[9];
    }
    atomicAdd(&p.stats->step_attempts, c_att);
    atomicAdd(&p.stats->rejected_steps, c_rej);
    atomicAdd(&p.stats->escape_substeps, c_esc);
    atomicAdd(&p.stats->rays, c_rays);
    atomicAdd(&p.stats->nan_rays, c_nan);
}

cudaError_t launch_plain(const KParams& p, int grid, int block, cudaStream_t stream) {
    void* args[] = {(void*)&p};
    const void* fn;
    switch (p.sc.kind) {
    case RTW_SCENE_MINKOWSKI_SPHERE: fn = (const void*)plain_kernel<RTW_SCENE_MINKOWSKI_SPHERE>; break;
    case RTW_SCENE_SCHWARZSCHILD_DISK: fn = (const void*)plain_kernel<RTW_SCENE_SCHWARZSCHILD_DISK>; break;
    case RTW_SCENE_KERR_DISK: fn = (const void*)plain_kernel<RTW_SCENE_KERR_DISK>; break;
    default: fn = (const void*)plain_kernel<RTW_SCENE_KERR_THICK_DISK>; break;
    }
    return cudaLaunchKernel(fn, dim3(grid), dim3(block), args, 0, stream);
}

}  // namespace rtw
