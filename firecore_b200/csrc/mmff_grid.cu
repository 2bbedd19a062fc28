// mmff_grid.cu -- one-time GridFF construction on the GPU (FP64).
//
//  1. node potentials of a rigid substrate, GridFF::evalBsplineRef semantics
//     with bUseEwald=false (cpp/common/molecular/GridFF.h:847-891):
//       Pauli   sum  sqrt(E0_j) * exp(-2 a (r - R0_j))      (evalGridFFPoint_Mors :582)
//       London  sum -2 sqrt(E0_j) * exp(-a (r - R0_j))
//       Coulomb sum  k_e Q_j / r                             (evalGridFFPoint_Coul :614)
//     Morse over the nPBC_mors images, Coulomb over the nPBC_coul images.
//  2. exact cubic B-spline interpolation coefficients: periodic tridiagonal
//     solves along x and y, and a solve with zero coefficients outside the
//     grid along z -- the fixed point the reference's damped-MD least-squares
//     fit (Bspline::fit3D_omp, cpp/common/math/Bspline_fit_3D.h:411-495, bPBC)
//     iterates towards.
//  3. packing to float4 (P, L, Q, 0), z fastest (GridFF::pack_Bspline_d,
//     GridFF.h:1203-1216).
#include <cuda_runtime.h>
#include <stdint.h>

namespace mmff {

#define MMFF_COULOMB_D 14.3996448915

// substrate atoms in shared memory, tiles of 128
__global__ void grid_potential_kernel(int nx, int ny, int nz, double3 pos0, double3 step, int nsub,
                                      const double4* __restrict__ sposq,   // (x, y, z, Q)
                                      const double2* __restrict__ sRE,     // (R0, sqrt(E0))
                                      const double3* __restrict__ shm, int nm,
                                      const double3* __restrict__ shc, int nc, double alpha, double* __restrict__ V) {
    const long ntot = (long)nx * ny * nz;
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    __shared__ double4 sa[128];
    __shared__ double2 sr[128];
    const bool valid = i < ntot;
    int iz = 0, iy = 0, ix = 0;
    if (valid) { iz = (int)(i % nz); iy = (int)((i / nz) % ny); ix = (int)(i / ((long)nz * ny)); }
    const double px = pos0.x + step.x * ix, py = pos0.y + step.y * iy, pz = pos0.z + step.z * iz;
    double vp = 0, vl = 0, vc = 0;
    for (int t0 = 0; t0 < nsub; t0 += 128) {
        __syncthreads();
        if (t0 + (int)threadIdx.x < nsub && threadIdx.x < 128) { sa[threadIdx.x] = sposq[t0 + threadIdx.x]; sr[threadIdx.x] = sRE[t0 + threadIdx.x]; }
        __syncthreads();
        const int nt = min(128, nsub - t0);
        if (!valid) continue;
        for (int a = 0; a < nt; a++) {
            const double4 s = sa[a];
            const double2 r = sr[a];
            const double dx0 = px - s.x, dy0 = py - s.y, dz0 = pz - s.z;
            for (int k = 0; k < nm; k++) {
                const double3 sh = shm[k];
                const double dx = dx0 + sh.x, dy = dy0 + sh.y, dz = dz0 + sh.z;
                const double rr = sqrt(dx * dx + dy * dy + dz * dz + 1e-32);
                const double e = exp(-alpha * (rr - r.x));
                const double eM = e * r.y;
                vp += eM * e;
                vl += eM * -2.0;
            }
            double qsum = 0.0;
            for (int k = 0; k < nc; k++) {
                const double3 sh = shc[k];
                const double dx = dx0 + sh.x, dy = dy0 + sh.y, dz = dz0 + sh.z;
                qsum += rsqrt(dx * dx + dy * dy + dz * dz + 1e-32);
            }
            vc += MMFF_COULOMB_D * s.w * qsum;
        }
    }
    if (valid) { V[3 * i] = vp; V[3 * i + 1] = vl; V[3 * i + 2] = vc; }
}

// (c[i-1] + 4c[i] + c[i+1]) / 6 = v[i], zero outside [0, n): one thread per line
__global__ void solve_open_kernel(double* __restrict__ C, long nlines, int n, long line_stride, long elem_stride,
                                  int nlines_inner, long inner_stride, double* __restrict__ work) {
    const long l = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (l >= nlines) return;
    const long base = (l / nlines_inner) * line_stride + (l % nlines_inner) * inner_stride;
    double* cp = work + l * n;
    const double a = 1.0 / 6.0, b = 4.0 / 6.0;
    for (int ch = 0; ch < 3; ch++) {
        double* y = C + ch;
        cp[0] = a / b;
        y[3 * base] = y[3 * base] / b;
        for (int i = 1; i < n; i++) {
            const double diag = b - a * cp[i - 1];
            cp[i] = a / diag;
            const long k = base + i * elem_stride, km = base + (i - 1) * elem_stride;
            y[3 * k] = (y[3 * k] - a * y[3 * km]) / diag;
        }
        for (int i = n - 2; i >= 0; i--) {
            const long k = base + i * elem_stride, kp = base + (i + 1) * elem_stride;
            y[3 * k] -= cp[i] * y[3 * kp];
        }
    }
}

// periodic version (Sherman-Morrison on the cyclic tridiagonal system)
__global__ void solve_periodic_kernel(double* __restrict__ C, long nlines, int n, long line_stride, long elem_stride,
                                      int nlines_inner, long inner_stride, double* __restrict__ work) {
    const long l = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (l >= nlines) return;
    const long base = (l / nlines_inner) * line_stride + (l % nlines_inner) * inner_stride;
    double* cp = work + l * 2 * n;
    double* z = cp + n;
    const double a = 1.0 / 6.0, b = 4.0 / 6.0;
    const double gamma = -b;
    const double bb0 = b - gamma, bbn = b - a * a / gamma;
    // z = T^-1 u, u = (gamma, 0, ..., 0, a); it does not depend on the channel
    {
        cp[0] = a / bb0;
        z[0] = gamma / bb0;
        for (int i = 1; i < n; i++) {
            const double diag = (i == n - 1 ? bbn : b) - a * cp[i - 1];
            cp[i] = a / diag;
            const double ui = (i == n - 1) ? a : 0.0;
            z[i] = (ui - a * z[i - 1]) / diag;
        }
        for (int i = n - 2; i >= 0; i--) z[i] -= cp[i] * z[i + 1];
    }
    const double zden = 1.0 + z[0] + a * z[n - 1] / gamma;
    for (int ch = 0; ch < 3; ch++) {
        double* y = C + ch;
        y[3 * base] = y[3 * base] / bb0;
        for (int i = 1; i < n; i++) {
            const double diag = (i == n - 1 ? bbn : b) - a * cp[i - 1];
            const long k = base + i * elem_stride, km = base + (i - 1) * elem_stride;
            y[3 * k] = (y[3 * k] - a * y[3 * km]) / diag;
        }
        for (int i = n - 2; i >= 0; i--) {
            const long k = base + i * elem_stride, kp = base + (i + 1) * elem_stride;
            y[3 * k] -= cp[i] * y[3 * kp];
        }
        const long klast = base + (long)(n - 1) * elem_stride;
        const double fact = (y[3 * base] + a * y[3 * klast] / gamma) / zden;
        for (int i = 0; i < n; i++) y[3 * (base + i * elem_stride)] -= fact * z[i];
    }
}

__global__ void pack_grid_kernel(long ntot, const double* __restrict__ C, float4* __restrict__ G) {
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < ntot) G[i] = make_float4((float)C[3 * i], (float)C[3 * i + 1], (float)C[3 * i + 2], 0.f);
}

}  // namespace mmff
