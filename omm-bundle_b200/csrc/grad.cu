// Derivatives of the Kim functional and of the converged OMM energy.
//
// Functional gradient (libOMM's calc_G, omm_ops.F90:17-39): for
//     Omega(C) = tr[(2I - S_W) H_W],  H_W = C H C^H,  S_W = C S C^H,
// dOmega/dC = G = 4 HC - 2 S_W HC - 2 H_W SC  (HC = C H, SC = C S).
//
// Energy adjoint: the converged energy E(theta) = min_C Omega(C; H(theta))
// with H(theta) = H0 + sum_k theta_k V_k is stationary in C, so
//     dE/dtheta_k = dOmega/dtheta_k |_{C*} = Re sum_ij conj(D_ij) (V_k)_ij,
//     D = C^H (2I - S_W) C
// (the density matrix that omm() returns, omm.F90:575-582).  D is m x m and
// dense; the adjoint never forms it.  With CD = (2I - S_W) C (n x m),
//     conj(D_ij) = sum_a C_ai conj(CD_aj),
// so each nonzero (i, j, v) of V_k contributes v * <C(:,i), conj(CD(:,j))>:
// a sampled dense-dense product over the sparsity of V_k (SDDMM).  The kernel
// below takes one column j of V per CTA, keeps CD(:,j) in shared memory and
// lets each warp reduce the dot products of that column's nonzeros.
#include "internal.h"

#include <cmath>

namespace ommgpu {

namespace {

const double ONE[2] = {1.0, 0.0}, ZERO[2] = {0.0, 0.0}, MONE[2] = {-1.0, 0.0};

DView make_view(DevBuf& b, int rows, int cols, bool real) {
    b.alloc_zero(std::max<size_t>(1, (size_t)rows * cols) * (real ? 8 : 16));
    return DView{b.p, rows, cols, std::max(1, rows), real};
}

// A * M for M = H or S (dense or CSC); out n x m
void apply(const DView& A, const msw_matrix* M, DView& out, int m) {
    if (M->dense()) {
        Staged s;
        stage_in(M, s);
        gemm('n', 'n', A.rows, m, m, ONE, A, s.v, ZERO, out);
        sync();
    } else {
        spmm_dense_csc(A, M, out, ONE, ZERO);
    }
}

constexpr int kAdjThreads = 256;

// grad partial per CTA: sum over nonzeros (i, v) of column j of V of
// Re( v * sum_a C(a,i) * conj(CD(a,j)) ).
template <bool REAL>
__global__ void __launch_bounds__(kAdjThreads) adjoint_sddmm_kernel(int n, const double* __restrict__ C, int ldc,
                                                                   const double* __restrict__ CD, int ldcd,
                                                                   const int* __restrict__ colptr,
                                                                   const int* __restrict__ rowind,
                                                                   const double* __restrict__ val, double* part) {
    extern __shared__ double s_cd[];  // n (real) or 2n (complex) values of CD(:, j)
    const int j = blockIdx.x;
    const int w = REAL ? 1 : 2;
    for (int a = threadIdx.x; a < n * w; a += blockDim.x) s_cd[a] = CD[(size_t)j * ldcd * w + a];
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    double acc = 0.0;
    for (int l = colptr[j] + warp; l < colptr[j + 1]; l += nw) {
        const int i = rowind[l];
        const double* ci = C + (size_t)i * ldc * w;
        double re = 0.0, im = 0.0;
        if (REAL) {
            for (int a = lane; a < n; a += 32) re = fma(ci[a], s_cd[a], re);
        } else {
            for (int a = lane; a < n; a += 32) {
                double cr = ci[2 * a], cim = ci[2 * a + 1], dr = s_cd[2 * a], di = s_cd[2 * a + 1];
                re += cr * dr + cim * di;  // C * conj(CD)
                im += cim * dr - cr * di;
            }
        }
        for (int o = 16; o > 0; o >>= 1) {
            re += __shfl_down_sync(0xffffffffu, re, o);
            im += __shfl_down_sync(0xffffffffu, im, o);
        }
        if (lane == 0) {
            if (REAL) acc += val[l] * re;
            else acc += val[2 * l] * re - val[2 * l + 1] * im;  // Re(v * z)
        }
    }
    __shared__ double s_acc[kAdjThreads / 32];
    if (lane == 0) s_acc[warp] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int q = 0; q < nw; ++q) s += s_acc[q];
        part[j] = s;
    }
}

__global__ void sum_partials(const double* part, int n, double* out) {
    // deterministic single-block Neumaier sum
    __shared__ double ss[256], sc[256];
    double s = 0.0, c = 0.0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        double v = part[i], t = s + v;
        c += (fabs(s) >= fabs(v)) ? ((s - t) + v) : ((v - t) + s);
        s = t;
    }
    ss[threadIdx.x] = s;
    sc[threadIdx.x] = c;
    __syncthreads();
    if (threadIdx.x == 0) {
        double S = 0.0, Cc = 0.0;
        for (int i = 0; i < (int)blockDim.x; ++i) {
            double v = ss[i], t = S + v;
            Cc += (fabs(S) >= fabs(v)) ? ((S - t) + v) : ((v - t) + S);
            S = t;
            Cc += sc[i];
        }
        *out = S + Cc;
    }
}

}  // namespace

// d E / d theta for one sparse perturbation, given C and CD = (2I - S_W) C on the device.
double adjoint_sparse(const DView& C, const DView& CD, const msw_matrix* V) {
    ensure_csc_device(V);
    int m = V->dim2, n = C.rows;
    DevBuf part;
    part.alloc_zero((size_t)(m + 1) * sizeof(double));
    size_t smem = (size_t)n * (C.is_real ? 8 : 16);
    if (smem > 200 * 1024) fail(OMM_ERR_UNSUPPORTED, "energy adjoint: n too large for one CD column in shared memory");
    // the kernel's static shared memory comes on top of the column: opt in for every size
    if (C.is_real)
        OMM_CK(cudaFuncSetAttribute(adjoint_sddmm_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    else
        OMM_CK(cudaFuncSetAttribute(adjoint_sddmm_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    if (C.is_real)
        adjoint_sddmm_kernel<true><<<m, kAdjThreads, smem, rt().stream>>>(n, (const double*)C.p, C.ld,
                                                                          (const double*)CD.p, CD.ld,
                                                                          V->d_colptr.as<int>(), V->d_rowind.as<int>(),
                                                                          V->d_val.as<double>(), part.as<double>());
    else
        adjoint_sddmm_kernel<false><<<m, kAdjThreads, smem, rt().stream>>>(n, (const double*)C.p, C.ld,
                                                                           (const double*)CD.p, CD.ld,
                                                                           V->d_colptr.as<int>(), V->d_rowind.as<int>(),
                                                                           V->d_val.as<double>(), part.as<double>());
    OMM_KCHECK();
    sum_partials<<<1, 256, 0, rt().stream>>>(part.as<double>(), m, part.as<double>() + m);
    OMM_KCHECK();
    double h = 0.0;
    OMM_CK(cudaMemcpyAsync(&h, part.as<double>() + m, sizeof(double), cudaMemcpyDeviceToHost, rt().stream));
    sync();
    return h;
}

}  // namespace ommgpu

using namespace ommgpu;

extern "C" {

int omm_gpu_functional_grad(int m, int n, const msw_matrix* H, const msw_matrix* S, const msw_matrix* C,
                            msw_matrix* G, double* omega) {
    try {
        if (!H || !C || !G || !omega) fail(OMM_ERR_ARG, "functional_grad: null argument");
        bool real = C->is_real;
        if (C->dim1 != n || C->dim2 != m || G->dim1 != n || G->dim2 != m || H->dim1 != m || H->dim2 != m)
            fail(OMM_ERR_ARG, "functional_grad: dimensions do not match");
        if (S && (S->dim1 != m || S->dim2 != m)) fail(OMM_ERR_ARG, "functional_grad: S has wrong dimensions");
        Staged sc, sg;
        stage_in(C, sc, true);
        stage_in(G, sg, false);
        DevBuf bHC, bSC, bHW, bSW, bT;
        DView HC = make_view(bHC, n, m, real), SC = make_view(bSC, n, m, real);
        DView HW = make_view(bHW, n, n, real), SW = make_view(bSW, n, n, real);
        apply(sc.v, H, HC, m);
        if (S) apply(sc.v, S, SC, m);
        else k_axpby(sc.v, 'n', SC, ONE, ZERO);
        gemm('n', 'c', n, n, m, ONE, HC, sc.v, ZERO, HW);
        gemm('n', 'c', n, n, m, ONE, SC, sc.v, ZERO, SW);
        double trh[2], trhs[2];
        r_trace(HW, trh);
        r_dot(HW, SW, trhs);
        *omega = 2.0 * trh[0] - trhs[0];  // coeff(0), omm_ops.F90:213
        double four[2] = {4.0, 0.0}, mtwo[2] = {-2.0, 0.0};
        k_axpby(HC, 'n', sg.v, four, ZERO);                 // G = 4 HC
        gemm('n', 'n', n, m, n, mtwo, SW, HC, ONE, sg.v);   // G -= 2 SW HC
        gemm('n', 'n', n, m, n, mtwo, HW, SC, ONE, sg.v);   // G -= 2 HW SC
        stage_out(G, sg);
        sync();
    } catch (const Error& e) {
        set_last_error(e.msg);
        return e.code;
    }
    set_last_error("");
    return OMM_OK;
}

int omm_gpu_energy_adjoint(int m, int n, const msw_matrix* S, const msw_matrix* C, int nv, const msw_matrix* const* V,
                           double* grad) {
    try {
        if (!C || (nv > 0 && (!V || !grad))) fail(OMM_ERR_ARG, "energy_adjoint: null argument");
        if (C->dim1 != n || C->dim2 != m) fail(OMM_ERR_ARG, "energy_adjoint: C must be n x m");
        bool real = C->is_real;
        Staged sc;
        stage_in(C, sc, true);
        DevBuf bSC, bSW, bQ, bCD;
        DView SC = make_view(bSC, n, m, real), SW = make_view(bSW, n, n, real);
        DView Q = make_view(bQ, n, n, real), CD = make_view(bCD, n, m, real);
        if (S) apply(sc.v, S, SC, m);
        else k_axpby(sc.v, 'n', SC, ONE, ZERO);
        gemm('n', 'c', n, n, m, ONE, SC, sc.v, ZERO, SW);   // S_W = C S C^H
        double two[2] = {2.0, 0.0};
        k_set(Q, 'a', ZERO, two);
        k_axpby(SW, 'n', Q, MONE, ONE);                     // Q = 2I - S_W
        gemm('n', 'n', n, m, n, ONE, Q, sc.v, ZERO, CD);    // CD = Q C
        for (int k = 0; k < nv; ++k) {
            const msw_matrix* Vk = V[k];
            if (!Vk || Vk->dim1 != m || Vk->dim2 != m || Vk->is_real != real)
                fail(OMM_ERR_ARG, "energy_adjoint: V_k must be m x m with the type of C");
            if (Vk->dense()) {
                // dense V: tr(Q C V C^H) through two GEMMs
                DevBuf bCV, bW;
                DView CV = make_view(bCV, n, m, real), W = make_view(bW, n, n, real);
                Staged sv;
                stage_in(Vk, sv);
                gemm('n', 'n', n, m, m, ONE, sc.v, sv.v, ZERO, CV);
                gemm('n', 'c', n, n, m, ONE, CV, sc.v, ZERO, W);
                double t[2];
                r_dot(Q, W, t);
                grad[k] = t[0];
            } else {
                grad[k] = adjoint_sparse(sc.v, CD, Vk);
            }
        }
        sync();
    } catch (const Error& e) {
        set_last_error(e.msg);
        return e.code;
    }
    set_last_error("");
    return OMM_OK;
}

}  // extern "C"
