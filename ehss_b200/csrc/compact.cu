// Isotropic incidence on compact enclosing boundaries (sphere, ellipsoid,
// box): CompactBoundary.source, src/support_exchange_transport/
// ehss_compact_source.py:47-87.  One thread per ray; FP64 in the reference's
// operation order with explicitly rounded intrinsics.  Transcendentals are
// CUDA's cos/sin (within 2 ulp of numpy's); the 3x3 products use the plain
// row order (the reference's numpy matmul may round differently in the last
// bit for a general rotation; the box boundary's rotation is the identity,
// where every order is exact).
#include "ehss_internal.cuh"

namespace ehss {

namespace {

constexpr double kTwoPi = 2.0 * 3.141592653589793;
constexpr double kPiD = 3.141592653589793;

// unit_sphere (inside_out_pa.py:45-49)
__device__ __forceinline__ void unit_sphere64(double u0, double u1, double* d) {
    double z = dsub(1.0, dmul(2.0, u0));
    double phi = dmul(kTwoPi, u1);
    double rho = dsqrt(dmax0(dsub(1.0, dmul(z, z))));
    double sp, cp;
    sincos(phi, &sp, &cp);
    d[0] = dmul(rho, cp); d[1] = dmul(rho, sp); d[2] = z;
}

// tangent_frames (inside_out_pa.py:52-58)
__device__ __forceinline__ void tangent_frames64(const double* d, double* t, double* b) {
    double a0 = 0., a1 = 0., a2 = 1.;
    if (fabs(d[2]) > .9) { a0 = 1.; a2 = 0.; }
    t[0] = dsub(dmul(a1, d[2]), dmul(a2, d[1]));
    t[1] = dsub(dmul(a2, d[0]), dmul(a0, d[2]));
    t[2] = dsub(dmul(a0, d[1]), dmul(a1, d[0]));
    double tn = dsqrt(dadd(dadd(dmul(t[0], t[0]), dmul(t[1], t[1])), dmul(t[2], t[2])));
    t[0] = ddiv(t[0], tn); t[1] = ddiv(t[1], tn); t[2] = ddiv(t[2], tn);
    b[0] = dsub(dmul(d[1], t[2]), dmul(d[2], t[1]));
    b[1] = dsub(dmul(d[2], t[0]), dmul(d[0], t[2]));
    b[2] = dsub(dmul(d[0], t[1]), dmul(d[1], t[0]));
}

// row vector v times the 3x3 matrix R (row major): (v R)_j = (v0 R0j + v1 R1j) + v2 R2j
__device__ __forceinline__ double vec_mat(const double* v, const double* R, int j) {
    return dadd(dadd(dmul(v[0], R[j]), dmul(v[1], R[3 + j])), dmul(v[2], R[6 + j]));
}

__device__ __forceinline__ double sum3(double a, double b, double c) { return dadd(dadd(a, b), c); }

}  // namespace

__global__ void k_compact_rays(ehss_boundary B, SobolParams p, int dim, int64_t first, int64_t n, double inv_count,
                               double* O, double* D, double* Wt) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t idx = (uint32_t)(first + i);
    const uint32_t g = idx ^ (idx >> 1);
    double u[5];
    for (int j = 0; j < dim; ++j) {
        uint32_t v = p.shift[j];
        uint32_t gg = g;
        while (gg) {
            int k = __ffs(gg) - 1;
            gg &= gg - 1;
            v ^= p.sv[j * 30 + k];
        }
        u[j] = (double)v * 0x1p-30;
    }
    double d[3], o[3], area;
    unit_sphere64(u[0], u[1], d);
    const double* c = B.center;
    const double* R = B.rotation;
    const double* ax = B.axes;
    if (B.kind == EHSS_BOUNDARY_SPHERE) {
        double t[3], b[3];
        tangent_frames64(d, t, b);
        const double radius = ax[0];
        const double rho = dmul(radius, dsqrt(u[2]));
        double ps, pc;
        sincos(dmul(kTwoPi, u[3]), &ps, &pc);
        for (int k = 0; k < 3; ++k)
            o[k] = dadd(dsub(c[k], dmul(radius, d[k])), dmul(rho, dadd(dmul(pc, t[k]), dmul(ps, b[k]))));
        area = dmul(dmul(kPiD, radius), radius);
    } else if (B.kind == EHSS_BOUNDARY_BOX) {
        double ld[3], proj[3], pt[3];
        for (int j = 0; j < 3; ++j) ld[j] = vec_mat(d, R, j);
        const double prod = dmul(dmul(ax[0], ax[1]), ax[2]);
        for (int j = 0; j < 3; ++j) proj[j] = dmul(fabs(ld[j]), ddiv(dmul(4.0, prod), ax[j]));
        area = sum3(proj[0], proj[1], proj[2]);
        // face k with probability proj[k] / area: count of running sums <= u2 * area
        const double x = dmul(u[2], area);
        const double c0 = proj[0], c1 = dadd(proj[0], proj[1]), c2 = dadd(c1, proj[2]);
        const int face = (x >= c0) + (x >= c1) + (x >= c2);
        const int f = face < 3 ? face : 2;
        const double sgn = ld[f] > 0. ? 1. : (ld[f] < 0. ? -1. : 0.);
        pt[f] = dmul(-sgn, ax[f]);
        int q = 3;
        for (int k = 0; k < 3; ++k)
            if (k != f) { pt[k] = dmul(dsub(dmul(2.0, u[q]), 1.0), ax[k]); ++q; }
        const double amax = fmax(fmax(ax[0], ax[1]), ax[2]);
        const double s = dmul(1e-10, fmax(1.0, amax));
        for (int k = 0; k < 3; ++k) {
            // (p R^T)_k = sum_j p_j R[k][j]
            double w = dadd(dadd(dmul(pt[0], R[3 * k]), dmul(pt[1], R[3 * k + 1])), dmul(pt[2], R[3 * k + 2]));
            o[k] = dsub(dadd(c[k], w), dmul(s, d[k]));
        }
    } else {   // ellipsoid
        double t[3], b[3], lt[3], lb[3], dv[3];
        tangent_frames64(d, t, b);
        for (int j = 0; j < 3; ++j) {
            lt[j] = dmul(vec_mat(t, R, j), ax[j]);
            lb[j] = dmul(vec_mat(b, R, j), ax[j]);
            dv[j] = dmul(vec_mat(d, R, j), ax[j]);
        }
        const double g00 = sum3(dmul(lt[0], lt[0]), dmul(lt[1], lt[1]), dmul(lt[2], lt[2]));
        const double g01 = sum3(dmul(lt[0], lb[0]), dmul(lt[1], lb[1]), dmul(lt[2], lb[2]));
        const double g11 = sum3(dmul(lb[0], lb[0]), dmul(lb[1], lb[1]), dmul(lb[2], lb[2]));
        const double l00 = dsqrt(g00);
        const double l10 = ddiv(g01, l00);
        const double l11 = dsqrt(dmax0(dsub(g11, dmul(l10, l10))));
        const double rho = dsqrt(u[2]);
        double ps, pc;
        sincos(dmul(kTwoPi, u[3]), &ps, &pc);
        const double x = dmul(rho, pc), y = dmul(rho, ps);
        const double e = dsqrt(sum3(dmul(dv[0], dv[0]), dmul(dv[1], dv[1]), dmul(dv[2], dv[2])));
        const double ee = dmul(e, 1.0 + 1e-10);
        const double a = dmul(l00, x), bb = dadd(dmul(l10, x), dmul(l11, y));
        for (int k = 0; k < 3; ++k) o[k] = dsub(dadd(c[k], dadd(dmul(a, t[k]), dmul(bb, b[k]))), dmul(ee, d[k]));
        area = dmul(dmul(kPiD, l00), l11);
    }
    for (int k = 0; k < 3; ++k) { O[3 * i + k] = o[k]; D[3 * i + k] = d[k]; }
    Wt[i] = dmul(area, inv_count);
}

int launch_compact_rays(const ehss_boundary& B, const SobolParams& p, int dim, int64_t first, int64_t n,
                        double inv_count, double* O, double* D, double* W, cudaStream_t stream) {
    if (n == 0) return EHSS_OK;
    k_compact_rays<<<(unsigned)((n + 127) / 128), 128, 0, stream>>>(B, p, dim, first, n, inv_count, O, D, W);
    return cuda_status(cudaGetLastError(), "compact source launch");
}

}  // namespace ehss
