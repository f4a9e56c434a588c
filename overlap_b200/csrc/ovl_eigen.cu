// Overlap eigenmodes in the U(1) background, the reference's production
// fermion start: InitialConditions::SetOverlapQEDEigenfunctions
// (INITIALCONDITIONS/FERMIONS/SetOverlapQEDEigenfunctions.cpp:5-86) with the
// Hamiltonian of OverlapQEDEigenfunctions::Setup
// (INITIALCONDITIONS/FERMIONS/BASIS/OverlapQEDEigenfunctions.cpp:141-591).
//
// The reference builds h_ov column by column -- an overlap application
// (Zolotarev rational sign function, multi-shift CG) per basis vector of a
// random orthonormal basis -- and diagonalises it with LAPACK's zheev.  Here
// the same operator is built densely and exactly on the device:
//   1. h_W = i D_W as a D x D matrix (D = 4 Nc V, index site + V (spin + 4 colour),
//      the reference's VectorIndex), D_W the Wilson operator of the links
//      ConvertU1GaugeLinks gives (:20-49): the U(1) phase in colour (0,0) --
//      1 for the z links, QED::GetUVal --, every other entry zero;
//   2. h_W = W diag(lambda) W^+ (cuSOLVER Xheevd), sign(h_W) = W diag(sign lambda) W^+
//      (one complex GEMM);
//   3. h_ov = M [(1 + m/2) g0 + (1 - m/2) sign(h_W)] (OverlapU.cpp:188-202 with
//      the exact sign function);
//   4. h_ov = V diag(omega) V^+ (Xheevd), ascending;
//   5. global mode g: particle g % 2, level g / 2; particles take the positive
//      eigenvalues from the smallest up, antiparticles the negative ones from
//      the one nearest zero down (BasisIndex D/2 - 1 - level, D/2 + level in the
//      reference's descending order, LapackDiagonalization.cpp:138-150);
//      psi = sqrt(V) v, psimid = psi e^{-i omega dt / 2}.
// The matrix assembly, the sign and combination kernels and the mode
// extraction are this file's; the two dense Hermitian diagonalisations (the
// reference's zheev) and the GEMM are cuSOLVER and cuBLAS calls.
#include <cublas_v2.h>
#include <cusolverDn.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "ovl_device.cuh"
#include "ovl_internal.h"
#include "ovl_stencil.cuh"

namespace ovl {

namespace {

// The links of the eigenmode problem: colour (0,0) the U(1) phase of (site,
// mu) (1 for mu = 2 or without a background), all other entries zero.
__device__ __forceinline__ cmat2<double> qed_link(const double2 *__restrict__ u1, int n01, int site, int mu) {
    cpx<double> ph = mk<double>(1.0, 0.0);
    if (u1 && mu < 2) {
        const double2 v = u1[2 * (site % n01) + mu];
        ph = mk<double>(v.x, v.y);
    }
    const cpx<double> z = mk<double>(0.0, 0.0);
    return cmat2<double>{ph, z, z, z};
}

// Column j of h_W at output site x: thread per (j, x).
__global__ void qed_hw_kernel(cpx<double> *__restrict__ H, const double2 *__restrict__ u1, Lattice L, double amass) {
    const int V = L.V, D = 4 * kColours * V, n01 = L.N0 * L.N1;
    const size_t n = (size_t)D * V;
    for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < n; t += (size_t)gridDim.x * blockDim.x) {
        const int x = (int)(t % V);
        const int j = (int)(t / V);
        const int sj = j % V, spin = (j / V) % 4, colour = j / (4 * V);
        Spinor<double> e, acc;
        for (int c = 0; c < kColours; c++)
            for (int a = 0; a < kSpin; a++) {
                e.c[c][a] = mk<double>(c == colour && a == spin ? 1.0 : 0.0, 0.0);
                acc.c[c][a] = mk<double>(x == sj && c == colour && a == spin ? amass : 0.0, 0.0);
            }
        const Nbrs nb = neighbours(L, x);
        if (nb.xp == sj) hop<double, 0, true>(acc, e, qed_link(u1, n01, x, 0));
        if (nb.xm == sj) hop<double, 0, false>(acc, e, qed_link(u1, n01, nb.xm, 0));
        if (nb.yp == sj) hop<double, 1, true>(acc, e, qed_link(u1, n01, x, 1));
        if (nb.ym == sj) hop<double, 1, false>(acc, e, qed_link(u1, n01, nb.ym, 1));
        if (nb.zp == sj) hop<double, 2, true>(acc, e, qed_link(u1, n01, x, 2));
        if (nb.zm == sj) hop<double, 2, false>(acc, e, qed_link(u1, n01, nb.zm, 2));
        for (int c = 0; c < kColours; c++)
            for (int a = 0; a < kSpin; a++) {
                const cpx<double> d = finish_component(acc.c[c][a], a);  // D = -i g0 / 2 (...)
                H[(size_t)(x + V * (a + 4 * c)) + (size_t)D * j] = mk<double>(-d.im, d.re);  // h_W = i D
            }
    }
}

// W_s = W diag(sign lambda): column j times the sign of its eigenvalue.
__global__ void sign_columns_kernel(const cpx<double> *__restrict__ W, const double *__restrict__ lambda,
                                    cpx<double> *__restrict__ Ws, int D, int *zero) {
    const size_t n = (size_t)D * D;
    for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < n; t += (size_t)gridDim.x * blockDim.x) {
        const int j = (int)(t / D);
        const double l = lambda[j];
        const double s = l > 0.0 ? 1.0 : (l < 0.0 ? -1.0 : 0.0);
        if (t % D == 0 && l == 0.0) atomicAdd(zero, 1);
        Ws[t] = mk<double>(s * W[t].re, s * W[t].im);
    }
}

// h_ov = M [(1 + m/2) g0 + (1 - m/2) S] in place of S.
__global__ void overlap_hamiltonian_kernel(cpx<double> *__restrict__ S, int D, int V, double mdw, double mf) {
    const size_t n = (size_t)D * D;
    const double cp = mdw * (1.0 + 0.5 * mf), cm = mdw * (1.0 - 0.5 * mf);
    for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < n; t += (size_t)gridDim.x * blockDim.x) {
        const int r = (int)(t % D), j = (int)(t / D);
        cpx<double> v = mk<double>(cm * S[t].re, cm * S[t].im);
        if (r == j) v.re += ((r / V) % 4 < 2 ? cp : -cp);
        S[t] = v;
    }
}

// Modes [0, count) in the reference layout [mode][site][colour][spin] (psi and
// psimid) from the eigenvectors (columns of Vecs, ascending omega).
__global__ void qed_modes_kernel(const cpx<double> *__restrict__ Vecs, const double *__restrict__ omega, int D, int V,
                                 int first_mode, int count, double dt, double2 *__restrict__ psi,
                                 double2 *__restrict__ mid, int *bad) {
    const size_t n = (size_t)count * V * kColours * kSpin;
    const double nrm = sqrt((double)V);
    for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < n; t += (size_t)gridDim.x * blockDim.x) {
        const int a = (int)(t % kSpin);
        const int c = (int)((t / kSpin) % kColours);
        const int site = (int)((t / (kSpin * kColours)) % V);
        const int s = (int)(t / ((size_t)kSpin * kColours * V));
        const int g = first_mode + s, particle = g & 1, level = g >> 1;
        const int col = particle == 0 ? D / 2 + level : D / 2 - 1 - level;
        const double w = omega[col];
        if (site == 0 && c == 0 && a == 0 && ((particle == 0 && w < 0.0) || (particle == 1 && w > 0.0)))
            atomicAdd(bad, 1);  // the frequency check of SetOverlapQEDEigenfunctions.cpp:33-35
        const cpx<double> v = Vecs[(size_t)(site + V * (a + 4 * c)) + (size_t)D * col];
        const cpx<double> p = mk<double>(nrm * v.re, nrm * v.im);
        double sn, cs;
        sincos(-0.5 * w * dt, &sn, &cs);
        psi[t] = make_double2(p.re, p.im);
        mid[t] = make_double2(p.re * cs - p.im * sn, p.re * sn + p.im * cs);
    }
}

int grid_for(size_t n, int sm_count) { return (int)std::max<size_t>(1, std::min<size_t>((n + 255) / 256, 32 * (size_t)sm_count)); }

// Hermitian eigensystem of A (D x D, column-major, overwritten by the
// eigenvectors), eigenvalues ascending into w.
int heevd(cusolverDnHandle_t h, cpx<double> *A, double *w, int D, cudaStream_t stream) {
    cusolverDnParams_t params;
    if (cusolverDnCreateParams(&params) != CUSOLVER_STATUS_SUCCESS) return 1;
    size_t dev_bytes = 0, host_bytes = 0;
    int rc = 0;
    if (cusolverDnXsyevd_bufferSize(h, params, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER, D, CUDA_C_64F, A, D,
                                    CUDA_R_64F, w, CUDA_C_64F, &dev_bytes, &host_bytes) != CUSOLVER_STATUS_SUCCESS)
        rc = 1;
    void *dwork = nullptr;
    int *info = nullptr;
    std::vector<char> hwork(host_bytes > 0 ? host_bytes : 1);
    if (!rc && (cudaMalloc(&dwork, std::max<size_t>(dev_bytes, 1)) != cudaSuccess ||
                cudaMalloc(&info, sizeof(int)) != cudaSuccess))
        rc = 2;
    if (!rc && cusolverDnXsyevd(h, params, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER, D, CUDA_C_64F, A, D,
                                CUDA_R_64F, w, CUDA_C_64F, dwork, dev_bytes, hwork.data(), host_bytes,
                                info) != CUSOLVER_STATUS_SUCCESS)
        rc = 1;
    int hinfo = 0;
    if (!rc && cudaMemcpyAsync(&hinfo, info, sizeof(int), cudaMemcpyDeviceToHost, stream) == cudaSuccess &&
        cudaStreamSynchronize(stream) == cudaSuccess && hinfo != 0)
        rc = 3;
    if (dwork) cudaFree(dwork);
    if (info) cudaFree(info);
    cusolverDnDestroyParams(params);
    return rc;
}

}  // namespace

// Returns 0 on success, 1 on a library error, 2 out of memory, 3 when a
// diagonalisation did not converge.  omega_host (D, or null): eigenvalues of
// h_ov ascending; h_host (D x D column-major, or null): h_ov; *zero_modes:
// eigenvalues of h_W equal to zero (sign taken as 0); *bad: modes whose
// frequency has the wrong sign for their particle index.
int qed_eigenmodes(const double *u1, const Lattice &L, double amass, double mdw, double mf, double dt, int first_mode,
                   int count, double2 *psi_ref, double2 *mid_ref, double *omega_host, double *h_host, int *zero_modes,
                   int *bad, int sm_count, cudaStream_t stream) {
    const int V = L.V, D = 4 * kColours * V;
    const size_t nn = (size_t)D * D;
    cpx<double> *A = nullptr, *B = nullptr;
    double *w = nullptr;
    int *counters = nullptr;
    cusolverDnHandle_t sol = nullptr;
    cublasHandle_t blas = nullptr;
    int rc = 0;
    auto release = [&]() {
        if (A) cudaFree(A);
        if (B) cudaFree(B);
        if (w) cudaFree(w);
        if (counters) cudaFree(counters);
        if (sol) cusolverDnDestroy(sol);
        if (blas) cublasDestroy(blas);
    };
    if (cudaMalloc(&A, sizeof(cpx<double>) * nn) != cudaSuccess || cudaMalloc(&B, sizeof(cpx<double>) * nn) != cudaSuccess ||
        cudaMalloc(&w, sizeof(double) * D) != cudaSuccess || cudaMalloc(&counters, sizeof(int) * 2) != cudaSuccess) {
        cudaGetLastError();
        release();
        return 2;
    }
    if (cusolverDnCreate(&sol) != CUSOLVER_STATUS_SUCCESS || cublasCreate(&blas) != CUBLAS_STATUS_SUCCESS ||
        cusolverDnSetStream(sol, stream) != CUSOLVER_STATUS_SUCCESS || cublasSetStream(blas, stream) != CUBLAS_STATUS_SUCCESS) {
        release();
        return 1;
    }
    cudaMemsetAsync(counters, 0, sizeof(int) * 2, stream);
    // 1. h_W, 2. its eigensystem and sign(h_W) = W_s W^+
    qed_hw_kernel<<<grid_for((size_t)D * V, sm_count), 256, 0, stream>>>(A, reinterpret_cast<const double2 *>(u1), L,
                                                                          amass);
    if ((rc = heevd(sol, A, w, D, stream))) {
        release();
        return rc;
    }
    sign_columns_kernel<<<grid_for(nn, sm_count), 256, 0, stream>>>(A, w, B, D, counters);
    const cuDoubleComplex one = make_cuDoubleComplex(1.0, 0.0), zero = make_cuDoubleComplex(0.0, 0.0);
    cpx<double> *S = nullptr;
    if (cudaMalloc(&S, sizeof(cpx<double>) * nn) != cudaSuccess) {
        cudaGetLastError();
        release();
        return 2;
    }
    if (cublasZgemm(blas, CUBLAS_OP_N, CUBLAS_OP_C, D, D, D, &one, reinterpret_cast<cuDoubleComplex *>(B), D,
                    reinterpret_cast<cuDoubleComplex *>(A), D, &zero, reinterpret_cast<cuDoubleComplex *>(S),
                    D) != CUBLAS_STATUS_SUCCESS) {
        cudaFree(S);
        release();
        return 1;
    }
    // 3. h_ov, 4. its eigensystem
    overlap_hamiltonian_kernel<<<grid_for(nn, sm_count), 256, 0, stream>>>(S, D, V, mdw, mf);
    if (h_host && cudaMemcpyAsync(h_host, S, sizeof(cpx<double>) * nn, cudaMemcpyDeviceToHost, stream) != cudaSuccess)
        rc = 1;
    if (!rc) rc = heevd(sol, S, w, D, stream);
    // 5. the modes
    if (!rc && count > 0)
        qed_modes_kernel<<<grid_for((size_t)count * V * 8, sm_count), 256, 0, stream>>>(
            S, w, D, V, first_mode, count, dt, psi_ref, mid_ref, counters + 1);
    int hc[2] = {0, 0};
    if (!rc && omega_host && cudaMemcpyAsync(omega_host, w, sizeof(double) * D, cudaMemcpyDeviceToHost, stream) != cudaSuccess)
        rc = 1;
    if (!rc && (cudaMemcpyAsync(hc, counters, sizeof(int) * 2, cudaMemcpyDeviceToHost, stream) != cudaSuccess ||
                cudaStreamSynchronize(stream) != cudaSuccess))
        rc = 1;
    if (zero_modes) *zero_modes = hc[0];
    if (bad) *bad = hc[1];
    cudaFree(S);
    release();
    return rc;
}

}  // namespace ovl
