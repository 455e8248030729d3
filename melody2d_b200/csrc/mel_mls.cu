// Gauss-point shape functions on the device: the moving-least-squares (MLS) pass of the reference's
// pre-processor -- linear basis (Preprocessor/MLS2DWithDerivatives.m:65-165), cubic-spline weight W1
// and its gradient (Preprocessor/WeightW1WithDerivatives.m:17-47), support rule |x_p - x_i| < r_i
// (Preprocessor/SupportDomain.m:16-18), supports listed in ascending node order -- for the points of
// many bodies in one launch.
//
// One CTA per body stages the body's nodes and radii in shared memory; one warp per Gauss point
// scans them 32 at a time, and a ballot per block of 32 nodes yields the supports already in
// ascending order.  Each lane adds the moment matrix terms of its supports, a fixed shuffle tree
// combines them, every lane solves the 3x3 system, and each lane writes the shape function and
// derivatives of its supports at positions given by the ballot prefix.  Two passes: counts, then
// (after an exclusive scan into the CSR offsets) the values.
//
// Arithmetic: the basis is centred on the evaluation point and scaled by the body's largest radius,
// p_k = (1, (x_k - x_p)/s, (y_k - y_p)/s), so the moment matrix is O(1) and well conditioned; the
// shape functions are invariant under that change of origin and scale, and the system is solved by
// Cholesky (the moment matrix is symmetric positive definite whenever three supports are not
// collinear).  Results agree with an LU solve in the pre-processor's global basis to the latter's
// conditioning, and they satisfy the linear reproducing conditions to round-off.
#include <cstdio>
#include <vector>
#include "mel_internal.h"

namespace {

constexpr int MLS_THREADS = 256;
constexpr int MLS_MAX_NODES = 4096;

// W1 and its gradient with respect to the point, rel = x_p - x_node, d = the node's radius
// (Preprocessor/WeightW1WithDerivatives.m:25-44)
__device__ __forceinline__ void weight_w1(double rx, double ry, double d, double& w, double& wx, double& wy)
{
    const double rho = sqrt(rx * rx + ry * ry);
    const double r = rho / d;
    if (r <= 0.5) {
        w = (2.0 / 3.0) - 4.0 * r * r + 4.0 * r * r * r;
        const double d3 = d * d * d;
        wx = (-8.0 * d * rx + 12.0 * rx * rho) / d3;
        wy = (-8.0 * d * ry + 12.0 * ry * rho) / d3;
    } else if (r <= 1.0) {
        w = (4.0 / 3.0) - 4.0 * r + 4.0 * r * r - (4.0 / 3.0) * r * r * r;
        const double fac = 4.0 * (-1.0 + 2.0 * r - r * r) / (r * d * d);
        wx = fac * rx;
        wy = fac * ry;
    } else {
        w = 0.; wx = 0.; wy = 0.;
    }
}

// solves L L^T x = b for the Cholesky factor of the symmetric 3x3 matrix a (a00 a01 a02 a11 a12 a22)
struct chol3 {
    double l00, l10, l20, l11, l21, l22;
    __device__ bool factor(const double* a)
    {
        l00 = sqrt(a[0]);
        l10 = a[1] / l00;
        l20 = a[2] / l00;
        l11 = sqrt(a[3] - l10 * l10);
        l21 = (a[4] - l20 * l10) / l11;
        l22 = sqrt(a[5] - l20 * l20 - l21 * l21);
        return l00 > 0. && l11 > 0. && l22 > 0. && isfinite(l22) && isfinite(l21);
    }
    __device__ void solve(const double* b, double* x) const
    {
        const double y0 = b[0] / l00;
        const double y1 = (b[1] - l10 * y0) / l11;
        const double y2 = (b[2] - l20 * y0 - l21 * y1) / l22;
        x[2] = y2 / l22;
        x[1] = (y1 - l21 * x[2]) / l11;
        x[0] = (y0 - l10 * x[1] - l20 * x[2]) / l00;
    }
};

// pass 0: support counts per point; pass 1: CSR values.  bad[0] receives 1 + the first point whose
// moment matrix is singular (fewer than three non-collinear supports)
__global__ void __launch_bounds__(MLS_THREADS) mls_kernel(int pass, const int* bnp, const double2* nodes,
                                                          const double* radii, const int* bpp, const double2* pts,
                                                          int* cnt, const long long* ptr, int* sidx, double* N,
                                                          double* Nx, double* Ny, int* bad)
{
    extern __shared__ double2 smem_nodes[];
    const int b = blockIdx.x;
    const int n0 = bnp[b], nn = bnp[b + 1] - n0;
    const int p0 = bpp[b], np = bpp[b + 1] - p0;
    double2* sx = smem_nodes;
    double* sr = reinterpret_cast<double*>(sx + nn);
    __shared__ double s_scale;
    for (int i = threadIdx.x; i < nn; i += blockDim.x) { sx[i] = nodes[n0 + i]; sr[i] = radii[n0 + i]; }
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (warp == 0) {
        double m = 0.;
        for (int i = lane; i < nn; i += 32) m = fmax(m, sr[i]);
        for (int o = 16; o; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
        if (lane == 0) s_scale = m;
    }
    __syncthreads();
    const double s = s_scale, is = 1.0 / s;
    const unsigned lt = (1u << lane) - 1u;
    for (int p = warp; p < np; p += MLS_THREADS / 32) {
        const double2 xp = pts[p0 + p];
        if (pass == 0) {
            int c = 0;
            for (int base = 0; base < nn; base += 32) {
                const int j = base + lane;
                bool hit = false;
                if (j < nn) {
                    const double dx = xp.x - sx[j].x, dy = xp.y - sx[j].y;
                    hit = dx * dx + dy * dy - sr[j] * sr[j] < 0.;
                }
                c += __popc(__ballot_sync(0xffffffffu, hit));
            }
            if (lane == 0) cnt[p0 + p] = c;
            continue;
        }
        // moments A, Ax, Ay (6 entries each) of the lane's supports, then a fixed shuffle tree
        double m[18];
#pragma unroll
        for (int k = 0; k < 18; k++) m[k] = 0.;
        for (int base = 0; base < nn; base += 32) {
            const int j = base + lane;
            if (j < nn) {
                const double dx = xp.x - sx[j].x, dy = xp.y - sx[j].y;
                if (dx * dx + dy * dy - sr[j] * sr[j] < 0.) {
                    double w, wx, wy;
                    weight_w1(dx, dy, sr[j], w, wx, wy);
                    const double q1 = -dx * is, q2 = -dy * is;
                    const double pp[6] = { 1., q1, q2, q1 * q1, q1 * q2, q2 * q2 };
#pragma unroll
                    for (int k = 0; k < 6; k++) { m[k] += w * pp[k]; m[6 + k] += wx * pp[k]; m[12 + k] += wy * pp[k]; }
                }
            }
        }
#pragma unroll
        for (int k = 0; k < 18; k++)
            for (int o = 16; o; o >>= 1) m[k] += __shfl_xor_sync(0xffffffffu, m[k], o);
        chol3 L;
        if (!L.factor(m)) {
            if (lane == 0) atomicCAS(bad, 0, p0 + p + 1);
            continue;
        }
        // g1 = A^-1 c, g2 = A^-1 (dc/dx - Ax g1), g3 = A^-1 (dc/dy - Ay g1), c = p(x_p) = (1, 0, 0)
        const double c[3] = { 1., 0., 0. };
        double g1[3], g2[3], g3[3], r[3];
        L.solve(c, g1);
        const double* ax = m + 6;
        const double* ay = m + 12;
        r[0] = 0. - (ax[0] * g1[0] + ax[1] * g1[1] + ax[2] * g1[2]);
        r[1] = is - (ax[1] * g1[0] + ax[3] * g1[1] + ax[4] * g1[2]);
        r[2] = 0. - (ax[2] * g1[0] + ax[4] * g1[1] + ax[5] * g1[2]);
        L.solve(r, g2);
        r[0] = 0. - (ay[0] * g1[0] + ay[1] * g1[1] + ay[2] * g1[2]);
        r[1] = 0. - (ay[1] * g1[0] + ay[3] * g1[1] + ay[4] * g1[2]);
        r[2] = is - (ay[2] * g1[0] + ay[4] * g1[1] + ay[5] * g1[2]);
        L.solve(r, g3);
        long long pos = ptr[p0 + p];
        for (int base = 0; base < nn; base += 32) {
            const int j = base + lane;
            bool hit = false;
            double dx = 0., dy = 0.;
            if (j < nn) {
                dx = xp.x - sx[j].x; dy = xp.y - sx[j].y;
                hit = dx * dx + dy * dy - sr[j] * sr[j] < 0.;
            }
            const unsigned bal = __ballot_sync(0xffffffffu, hit);
            if (hit) {
                double w, wx, wy;
                weight_w1(dx, dy, sr[j], w, wx, wy);
                const double q1 = -dx * is, q2 = -dy * is;
                const double a1 = g1[0] + g1[1] * q1 + g1[2] * q2;
                const double a2 = g2[0] + g2[1] * q1 + g2[2] * q2;
                const double a3 = g3[0] + g3[1] * q1 + g3[2] * q2;
                const long long e = pos + __popc(bal & lt);
                sidx[e] = j;
                N[e] = a1 * w;
                Nx[e] = a2 * w + a1 * wx;
                Ny[e] = a3 * w + a1 * wy;
            }
            pos += __popc(bal);
        }
    }
}

// exclusive scan of n counts into out[0..n] (64-bit offsets), one block: n is a few million at most
__global__ void __launch_bounds__(1024) mls_scan_kernel(const int* cnt, long long* out, int n)
{
    __shared__ long long part[1024];
    const int t = threadIdx.x;
    const long long per = ((long long)n + 1023) / 1024;
    const long long a = t * per, e = min((long long)n, a + per);
    long long s = 0;
    for (long long i = a; i < e; i++) s += cnt[i];
    part[t] = s;
    __syncthreads();
    for (int o = 1; o < 1024; o <<= 1) {
        long long v = t >= o ? part[t - o] : 0;
        __syncthreads();
        part[t] += v;
        __syncthreads();
    }
    long long run = part[t] - s;
    for (long long i = a; i < e; i++) { out[i] = run; run += cnt[i]; }
    if (t == 1023) out[n] = part[1023];
}

template <typename T>
struct dbuf {
    T* p = nullptr;
    ~dbuf() { if (p) cudaFree(p); }
    cudaError_t alloc(size_t n) { return cudaMalloc(&p, sizeof(T) * (n ? n : 1)); }
};

}  // namespace

mel_status mel_mls_shapes(int n_bodies, const int* body_node_ptr, const double* nodes, const double* radii,
                          const int* body_point_ptr, const double* points, long long* sup_ptr, int* sup_idx,
                          double* N, double* dNdx, double* dNdy, long long capacity, long long* n_entries, int device,
                          double* kernel_ms)
{
    if (n_bodies <= 0 || !body_node_ptr || !nodes || !radii || !body_point_ptr || !points || !sup_ptr || !n_entries) {
        mel_set_error("invalid arguments");
        return MEL_ERR_INVALID;
    }
    const int nn = body_node_ptr[n_bodies], np = body_point_ptr[n_bodies];
    int max_nodes = 0;
    for (int b = 0; b < n_bodies; b++) {
        const int k = body_node_ptr[b + 1] - body_node_ptr[b];
        if (k < 0 || body_point_ptr[b + 1] < body_point_ptr[b]) { mel_set_error("body ranges must not decrease"); return MEL_ERR_INVALID; }
        max_nodes = k > max_nodes ? k : max_nodes;
    }
    if (max_nodes > MLS_MAX_NODES) { mel_set_error("a body has %d nodes (at most %d)", max_nodes, MLS_MAX_NODES); return MEL_ERR_UNSUPPORTED; }
    if (np == 0) { sup_ptr[0] = 0; *n_entries = 0; return MEL_OK; }
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) { mel_set_error("no CUDA device"); return MEL_ERR_NO_DEVICE; }
    MEL_CUDA_OK(cudaSetDevice(device));
    dbuf<int> d_bnp, d_bpp, d_cnt, d_bad, d_idx;
    dbuf<double2> d_nodes, d_pts;
    dbuf<double> d_r, d_N, d_Nx, d_Ny;
    dbuf<long long> d_ptr;
    MEL_CUDA_OK(d_bnp.alloc(n_bodies + 1)); MEL_CUDA_OK(d_bpp.alloc(n_bodies + 1));
    MEL_CUDA_OK(d_nodes.alloc(nn)); MEL_CUDA_OK(d_r.alloc(nn)); MEL_CUDA_OK(d_pts.alloc(np));
    MEL_CUDA_OK(d_cnt.alloc(np)); MEL_CUDA_OK(d_ptr.alloc((size_t)np + 1)); MEL_CUDA_OK(d_bad.alloc(1));
    MEL_CUDA_OK(cudaMemcpy(d_bnp.p, body_node_ptr, sizeof(int) * (n_bodies + 1), cudaMemcpyHostToDevice));
    MEL_CUDA_OK(cudaMemcpy(d_bpp.p, body_point_ptr, sizeof(int) * (n_bodies + 1), cudaMemcpyHostToDevice));
    MEL_CUDA_OK(cudaMemcpy(d_nodes.p, nodes, sizeof(double2) * nn, cudaMemcpyHostToDevice));
    MEL_CUDA_OK(cudaMemcpy(d_r.p, radii, sizeof(double) * nn, cudaMemcpyHostToDevice));
    MEL_CUDA_OK(cudaMemcpy(d_pts.p, points, sizeof(double2) * np, cudaMemcpyHostToDevice));
    MEL_CUDA_OK(cudaMemset(d_bad.p, 0, sizeof(int)));
    const size_t smem = (size_t)max_nodes * (sizeof(double2) + sizeof(double));
    MEL_CUDA_OK(cudaFuncSetAttribute(mls_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    mls_kernel<<<n_bodies, MLS_THREADS, smem>>>(0, d_bnp.p, d_nodes.p, d_r.p, d_bpp.p, d_pts.p, d_cnt.p, nullptr,
                                                 nullptr, nullptr, nullptr, nullptr, d_bad.p);
    MEL_CUDA_OK(cudaGetLastError());
    mls_scan_kernel<<<1, 1024>>>(d_cnt.p, d_ptr.p, np);
    MEL_CUDA_OK(cudaGetLastError());
    MEL_CUDA_OK(cudaMemcpy(sup_ptr, d_ptr.p, sizeof(long long) * ((size_t)np + 1), cudaMemcpyDeviceToHost));
    const long long ne = sup_ptr[np];
    *n_entries = ne;
    if (!sup_idx) return MEL_OK;                     // counting call
    if (capacity < ne || !N || !dNdx || !dNdy) {
        mel_set_error("output capacity %lld below the %lld support entries", capacity, ne);
        return MEL_ERR_INVALID;
    }
    MEL_CUDA_OK(d_idx.alloc(ne)); MEL_CUDA_OK(d_N.alloc(ne)); MEL_CUDA_OK(d_Nx.alloc(ne)); MEL_CUDA_OK(d_Ny.alloc(ne));
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (kernel_ms) { cudaEventCreate(&e0); cudaEventCreate(&e1); cudaEventRecord(e0); }
    mls_kernel<<<n_bodies, MLS_THREADS, smem>>>(1, d_bnp.p, d_nodes.p, d_r.p, d_bpp.p, d_pts.p, nullptr, d_ptr.p,
                                                 d_idx.p, d_N.p, d_Nx.p, d_Ny.p, d_bad.p);
    MEL_CUDA_OK(cudaGetLastError());
    if (kernel_ms) {
        // device time of the value pass (the count pass and the scan run before it)
        float ms = 0.f;
        cudaEventRecord(e1);
        cudaEventSynchronize(e1);
        cudaEventElapsedTime(&ms, e0, e1);
        *kernel_ms = ms;
        cudaEventDestroy(e0); cudaEventDestroy(e1);
    }
    int bad = 0;
    MEL_CUDA_OK(cudaMemcpy(&bad, d_bad.p, sizeof(int), cudaMemcpyDeviceToHost));
    if (bad) { mel_set_error("Gauss point %d has a singular moment matrix (fewer than three non-collinear supports)", bad - 1); return MEL_ERR_INVALID; }
    MEL_CUDA_OK(cudaMemcpy(sup_idx, d_idx.p, sizeof(int) * ne, cudaMemcpyDeviceToHost));
    MEL_CUDA_OK(cudaMemcpy(N, d_N.p, sizeof(double) * ne, cudaMemcpyDeviceToHost));
    MEL_CUDA_OK(cudaMemcpy(dNdx, d_Nx.p, sizeof(double) * ne, cudaMemcpyDeviceToHost));
    MEL_CUDA_OK(cudaMemcpy(dNdy, d_Ny.p, sizeof(double) * ne, cudaMemcpyDeviceToHost));
    return MEL_OK;
}
