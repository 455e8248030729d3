// Update_proximity (Code/Proximity.h:48-473) on the device.
//
// Stages (all integer bookkeeping deterministic, geometry bit-identical to the reference):
//   aabb_kernel       border boxes inflated by the detection distance and their period shifts
//                     (Code/Proximity.h:63-109), one warp per border
//   neighbour_kernel  all-pairs (body, border) overlap with periodic shifts and de-duplication
//                     (Code/Proximity.h:112-169), one warp per body, lanes over candidate bodies
//   [host]            task list: one task per (slave body, slave border, neighbour) in the
//                     reference's loop order, then one self task per (slave body, border)
//   count_kernel      accepted candidates per (task, slave border node) slot, one warp per task
//   scan              slot offsets = the canonical position of every new contact element
//   write_kernel      writes the new list in the reference's order; history inheritance searches the
//                     previous list of the same slave border node (Code/Proximity.h:269-284)
//   entry_index_kernel / incoming ranges   index structures for the next step and update
#include <cstdio>
#include <vector>
#include <algorithm>
#include "mel_internal.h"
#include "mel_geometry.cuh"

namespace mel {

// ---------------------------------------------------------------------------------------------
// exclusive scan of int (three-phase, deterministic)
// ---------------------------------------------------------------------------------------------
#define SCAN_BLOCK 1024
__global__ void scan_block_kernel(const int* in, int* out, int n, int* block_sums)
{
    __shared__ int s[SCAN_BLOCK];
    int i = blockIdx.x * SCAN_BLOCK + threadIdx.x;
    int v = (i < n) ? in[i] : 0;
    s[threadIdx.x] = v;
    __syncthreads();
    for (int off = 1; off < SCAN_BLOCK; off <<= 1) {
        int t = (threadIdx.x >= off) ? s[threadIdx.x - off] : 0;
        __syncthreads();
        s[threadIdx.x] += t;
        __syncthreads();
    }
    if (i <= n) out[i] = s[threadIdx.x] - v;
    if (threadIdx.x == SCAN_BLOCK - 1) block_sums[blockIdx.x] = s[threadIdx.x];
}
__global__ void scan_add_kernel(int* out, int n, const int* block_off)
{
    int i = blockIdx.x * SCAN_BLOCK + threadIdx.x;
    if (i < n) out[i] += block_off[blockIdx.x];   // n here counts the total slot as well
}

} // namespace mel

// out has n+1 entries: out[n] = total
void mel_scan_exclusive(const int* in, int* out, int n, cudaStream_t s)
{
    int nblk = (n + SCAN_BLOCK) / SCAN_BLOCK;   // covers index n as well
    int* sums = nullptr;
    int* soff = nullptr;
    cudaMallocAsync(&sums, sizeof(int) * (nblk + 1), s);
    cudaMallocAsync(&soff, sizeof(int) * (nblk + 2), s);
    mel::scan_block_kernel<<<nblk, SCAN_BLOCK, 0, s>>>(in, out, n, sums);
    if (nblk > 1) mel_scan_exclusive(sums, soff, nblk, s);
    else cudaMemsetAsync(soff, 0, sizeof(int), s);
    mel::scan_add_kernel<<<nblk, SCAN_BLOCK, 0, s>>>(out, n + 1, soff);
    cudaFreeAsync(sums, s);
    cudaFreeAsync(soff, s);
}

namespace mel {

// ---------------------------------------------------------------------------------------------
__global__ void aabb_kernel(mel_dev d, double* aabb, int* shmin, int* shmax)
{
    int g = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    int lane = threadIdx.x & 31;
    if (g >= d.nbd) return;
    int b = d.bd_body[g];
    if (d.b_status[b] == MEL_STATUS_INACTIVE) return;
    double dd = d.b_dist[3 * b + 1];
    int n0 = d.b_node0[b];
    double xmin = 1.e100, xmax = -1.e100, ymin = 1.e100, ymax = -1.e100;
    for (int e = d.bd_e0[g] + lane; e < d.bd_e0[g + 1]; e += 32) {
        double2 p = d.x[n0 + d.e_node[e]];
        if (p.x - dd < xmin) xmin = p.x - dd;
        if (p.x + dd > xmax) xmax = p.x + dd;
        if (p.y - dd < ymin) ymin = p.y - dd;
        if (p.y + dd > ymax) ymax = p.y + dd;
    }
    for (int o = 16; o > 0; o >>= 1) {
        xmin = fmin(xmin, __shfl_xor_sync(0xffffffffu, xmin, o));
        xmax = fmax(xmax, __shfl_xor_sync(0xffffffffu, xmax, o));
        ymin = fmin(ymin, __shfl_xor_sync(0xffffffffu, ymin, o));
        ymax = fmax(ymax, __shfl_xor_sync(0xffffffffu, ymax, o));
    }
    if (lane == 0) {
        double invperiod = 1. / d.period;
        aabb[4 * g] = xmin; aabb[4 * g + 1] = xmax; aabb[4 * g + 2] = ymin; aabb[4 * g + 3] = ymax;
        shmin[g] = (int)floor((xmin - d.xmin) * invperiod);
        shmax[g] = (int)floor((xmax - d.xmin) * invperiod);
    }
}

__global__ void neighbour_kernel(mel_dev d, const double* aabb, const int* shmin, const int* shmax,
                                 int* nbr, int* nbn, int cap)
{
    int b1 = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    int lane = threadIdx.x & 31;
    if (b1 >= d.nb) return;
    if (d.b_status[b1] == MEL_STATUS_INACTIVE) { if (lane == 0) nbn[b1] = 0; return; }
    int* out = nbr + (size_t)3 * cap * b1;
    int count = 0;
    for (int g1 = d.b_bd0[b1]; g1 < d.b_bd0[b1 + 1]; g1++) {
        double xmin1 = aabb[4 * g1], xmax1 = aabb[4 * g1 + 1], ymin1 = aabb[4 * g1 + 2], ymax1 = aabb[4 * g1 + 3];
        int smin1 = shmin[g1], smax1 = shmax[g1];
        int first_border = (g1 == d.b_bd0[b1]);
        int count_before = count;   // entries of earlier border1 iterations (dedup scope)
        for (int base = 0; base < d.nb; base += 32) {
            int b2 = base + lane;
            bool ok = b2 < d.nb && b2 != b1 && d.b_status[b2] != MEL_STATUS_INACTIVE;
            int mine = 0;
            for (int pass = 0; pass < 2; pass++) {
                int k = 0;
                if (ok) {
                    for (int g2 = d.b_bd0[b2]; g2 < d.b_bd0[b2 + 1]; g2++) {
                        double xmin2 = aabb[4 * g2], xmax2 = aabb[4 * g2 + 1], ymin2 = aabb[4 * g2 + 2], ymax2 = aabb[4 * g2 + 3];
                        if ((ymax2 < ymin1) || (ymax1 < ymin2)) continue;
                        int r2 = g2 - d.b_bd0[b2];
                        for (int s = smin1 - shmax[g2]; s <= smax1 - shmin[g2]; s++) {
                            if ((xmax2 + s * d.period > xmin1) && (xmin2 + s * d.period < xmax1)) {
                                bool dup = false;
                                if (!first_border) {
                                    for (int q = 0; q < count_before && q < cap; q++)
                                        if (out[3 * q] == b2 && out[3 * q + 1] == r2 && out[3 * q + 2] == s) { dup = true; break; }
                                }
                                if (dup) continue;
                                if (pass == 1) {
                                    int pos = mine + k;
                                    if (pos < cap) { out[3 * pos] = b2; out[3 * pos + 1] = r2; out[3 * pos + 2] = s; }
                                }
                                k++;
                            }
                        }
                    }
                }
                if (pass == 0) {
                    // exclusive prefix of k across lanes
                    int incl = k;
                    for (int o = 1; o < 32; o <<= 1) {
                        int t = __shfl_up_sync(0xffffffffu, incl, o);
                        if (lane >= o) incl += t;
                    }
                    int total = __shfl_sync(0xffffffffu, incl, 31);
                    mine = count + incl - k;
                    count += total;
                }
            }
            __syncwarp();
        }
    }
    if (lane == 0) {
        nbn[b1] = count;
        if (count > cap) { atomicOr(&d.err[MEL_E_NBR_OVERFLOW], 1u); atomicMax(&d.err[MEL_E_NBR_NEED], (unsigned)count); }
    }
}

// candidate enumeration shared by the count and write passes -----------------------------------
struct Cand {
    int seg, bM, rM, shM;
    Proj p;
    int nd[4], sh[4];
};

// regular task: slave node kS of global border gS of body bS against neighbour (bM, rM, shM)
template <typename F>
__device__ __forceinline__ void enum_regular(const mel_dev& d, int bS, int gS, int kS, int bM, int rM, int shM, F&& f)
{
    int gM = d.b_bd0[bM] + rM;
    int eM0 = d.bd_e0[gM], nM = d.bd_e0[gM + 1] - eM0;
    int eS = d.bd_e0[gS] + kS;
    double2 xs = d.x[d.b_node0[bS] + d.e_node[eS]];
    double dd = d.b_dist[3 * bS + 1], cd = d.b_dist[3 * bS + 2];
    int mb = d.b_node0[bM];
    for (int seg = 0; seg < nM - 1; seg++) {
        int e = eM0 + seg;
        const int* sn = d.e_sn + 4 * e;
        const int* ss = d.e_ss + 4 * e;
        double2 p1 = d.x[mb + sn[1]], p2 = d.x[mb + sn[2]];
        double X1 = p1.x + d.period * (shM + ss[1]), Y1 = p1.y;
        double X2 = p2.x + d.period * (shM + ss[2]), Y2 = p2.y;
        if (detect_proximity(xs.x, xs.y, X1, Y1, X2, Y2, dd) == 0) continue;
        double2 p0 = d.x[mb + sn[0]], p3 = d.x[mb + sn[3]];
        double X0 = p0.x + d.period * (shM + ss[0]), Y0 = p0.y;
        double X3 = p3.x + d.period * (shM + ss[3]), Y3 = p3.y;
        Proj p;
        p.gap = 0.; p.xsi = 0.; p.xn = p.yn = p.xt = p.yt = 0.; p.N[0] = p.N[1] = p.N[2] = p.N[3] = 0.; p.flag = 0;
        closest_linear(xs.x, xs.y, X0, Y0, X1, Y1, X2, Y2, X3, Y3, p);
        if ((p.flag == -2 || p.flag == -1 || p.flag == 0) && (p.gap > -cd)) f(seg, e, p);
    }
}

// self task: slave node kS of global border gS of body bS against the body's own segments
// (Code/Proximity.h:355-405); Closest_2_segment_self never yields flag 0, so those pairs are skipped
template <typename F>
__device__ __forceinline__ void enum_self(const mel_dev& d, int bS, int gS, int kS, F&& f)
{
    int eS = d.bd_e0[gS] + kS;
    int NodeS = d.e_node[eS];
    int n0 = d.b_node0[bS];
    double2 xs = d.x[n0 + NodeS];
    double dd = d.b_dist[3 * bS + 1], cd = d.b_dist[3 * bS + 2];
    for (int gM = d.b_bd0[bS]; gM < d.b_bd0[bS + 1]; gM++) {
        int eM0 = d.bd_e0[gM], nM = d.bd_e0[gM + 1] - eM0;
        for (int seg = 0; seg < nM - 1; seg++) {
            int e = eM0 + seg;
            const int* sn = d.e_sn + 4 * e;
            if (sn[1] == NodeS) continue;
            if (sn[2] == NodeS) continue;
            double2 p1 = d.x[n0 + sn[1]], p2 = d.x[n0 + sn[2]];
            if (detect_proximity(xs.x, xs.y, p1.x, p1.y, p2.x, p2.y, dd) == 0) continue;
            if (sn[0] == NodeS || sn[3] == NodeS) continue;
            double2 p0 = d.x[n0 + sn[0]], p3 = d.x[n0 + sn[3]];
            Proj p;
            p.gap = 0.; p.xsi = 0.; p.xn = p.yn = p.xt = p.yt = 0.; p.N[0] = p.N[1] = p.N[2] = p.N[3] = 0.; p.flag = 0;
            closest_linear(xs.x, xs.y, p0.x, p0.y, p1.x, p1.y, p2.x, p2.y, p3.x, p3.y, p);
            if (p.flag == 0 && (p.gap > -cd)) f(seg, e, p, gM - d.b_bd0[bS]);
        }
    }
}

__global__ void count_kernel(mel_dev d, const int* task, int ntask, const int* nbr, int cap, int* slot_cnt)
{
    int t = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    int lane = threadIdx.x & 31;
    if (t >= ntask) return;
    int bS = task[4 * t], gS = task[4 * t + 1], q = task[4 * t + 2], slot0 = task[4 * t + 3];
    int nS = d.bd_e0[gS + 1] - d.bd_e0[gS];
    for (int kS = lane; kS < nS; kS += 32) {
        int cnt = 0;
        if (q >= 0) {
            const int* nb = nbr + (size_t)3 * cap * bS + 3 * q;
            enum_regular(d, bS, gS, kS, nb[0], nb[1], nb[2], [&](int, int, const Proj&) { cnt++; });
        } else {
            enum_self(d, bS, gS, kS, [&](int, int, const Proj&, int) { cnt++; });
        }
        slot_cnt[slot0 + kS] = cnt;
    }
}

__global__ void write_kernel(mel_dev d, const int* task, int ntask, const int* nbr, int cap, const int* slot_off,
                             mel_contact* out, const mel_contact* old, const int* old_eptr, const int* old_elist,
                             int have_old)
{
    int t = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    int lane = threadIdx.x & 31;
    if (t >= ntask) return;
    int bS = task[4 * t], gS = task[4 * t + 1], q = task[4 * t + 2], slot0 = task[4 * t + 3];
    int rS = gS - d.b_bd0[bS];
    int eS0 = d.bd_e0[gS];
    int nS = d.bd_e0[gS + 1] - eS0;
    for (int kS = lane; kS < nS; kS += 32) {
        int pos = slot_off[slot0 + kS];
        int eS = eS0 + kS;
        int NodeS = d.e_node[eS];
        double length = d.e_len[eS];
        if (q >= 0) {
            const int* nb = nbr + (size_t)3 * cap * bS + 3 * q;
            int bM = nb[0], rM = nb[1], shM = nb[2];
            double effm;
            const double* rgM = d.rg + MEL_RIGID_NF * bM;
            const double* rgS = d.rg + MEL_RIGID_NF * bS;
            if (rgM[MEL_RG_MASS] == 0.) effm = 0.;
            else if (rgS[MEL_RG_MASS] == 0.) effm = 0.;
            else effm = 1. / (rgM[MEL_RG_INV_MASS] + rgS[MEL_RG_INV_MASS]);
            enum_regular(d, bS, gS, kS, bM, rM, shM, [&](int seg, int e, const Proj& p) {
                mel_contact c;
                bool found = false;
                if (have_old) {
                    for (int k = old_eptr[eS]; k < old_eptr[eS + 1]; k++) {
                        const mel_contact& o = old[old_elist[k]];
                        if (o.bodyM == bM && o.borderM == rM && abs(o.segmentM - seg) <= 1) { c = o; found = true; break; }
                    }
                }
                if (!found) {
                    c.bodyS = bS; c.borderS = rS; c.border_nodeS = kS; c.nodeS = NodeS;
                    c.bodyM = bM; c.borderM = rM; c.shiftM = shM; c.segmentM = seg;
                    for (int k = 0; k < 4; k++) { c.nodeM[k] = d.e_sn[4 * e + k]; c.shiftMk[k] = d.e_ss[4 * e + k]; c.shapeM[k] = p.N[k]; }
                    c.gapn = p.gap; c.vgapn = 0.; c.gapt = 0.; c.vgapt = 0.; c.xsi = p.xsi;
                    c.xnorm = p.xn; c.ynorm = p.yn; c.xtan = p.xt; c.ytan = p.yt;
                    c.effective_mass = effm; c.length = length; c.fx = 0.; c.fy = 0.;
                    c.nb_internal = 0; c.internal[0] = 0.; c.internal[1] = 0.; c.internal[2] = 0.;
                }
                c.bodyS = bS;
                c.pad_ = found ? 0 : 1;      // new elements get vgapn/vgapt in carry_kernel
                out[pos++] = c;
            });
        } else {
            double effm = d.rg[MEL_RIGID_NF * bS + MEL_RG_MASS];
            enum_self(d, bS, gS, kS, [&](int seg, int e, const Proj& p, int rM) {
                mel_contact c;
                c.bodyS = bS; c.borderS = rS; c.border_nodeS = kS; c.nodeS = NodeS;
                c.bodyM = bS; c.borderM = rM; c.shiftM = 0; c.segmentM = seg;
                for (int k = 0; k < 4; k++) { c.nodeM[k] = d.e_sn[4 * e + k]; c.shiftMk[k] = 0; c.shapeM[k] = p.N[k]; }
                c.gapn = p.gap; c.vgapn = 0.; c.gapt = 0.; c.vgapt = 0.; c.xsi = p.xsi;
                c.xnorm = p.xn; c.ynorm = p.yn; c.xtan = p.xt; c.ytan = p.yt;
                c.effective_mass = effm; c.length = length; c.fx = 0.; c.fy = 0.;
                c.nb_internal = 0; c.pad_ = 1; c.internal[0] = 0.; c.internal[1] = 0.; c.internal[2] = 0.;
                out[pos++] = c;
            });
        }
    }
}

// per-body serial counting sort of a body-major contact list by slave border entry
__global__ void entry_index_kernel(mel_dev d, const mel_contact* cont, const int* b_cont0, int* eptr_cnt, int* elist)
{
    int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= d.nb) return;
    int e_lo = d.bd_e0[d.b_bd0[b]], e_hi = d.bd_e0[d.b_bd0[b + 1]];
    int c0 = b_cont0[b], c1 = b_cont0[b + 1];
    // eptr_cnt holds the exclusive offsets of this body's entries (prepared by the caller);
    // fill in list order, advancing a per-entry cursor kept in elist space of the body
    for (int c = c0; c < c1; c++) {
        int e = d.bd_e0[d.b_bd0[b] + cont[c].borderS] + cont[c].border_nodeS;
        if (e < e_lo || e >= e_hi) { atomicOr(&d.err[MEL_E_BOUNDS], 2u); continue; }
        int slot = atomicAdd(&eptr_cnt[e], 1);   // only this thread touches the entries of body b
        elist[slot] = c;
    }
}

__global__ void entry_count_kernel(mel_dev d, const mel_contact* cont, int n, int* cnt)
{
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n) return;
    int b = cont[c].bodyS;
    int e = d.bd_e0[d.b_bd0[b] + cont[c].borderS] + cont[c].border_nodeS;
    atomicAdd(&cnt[e], 1);
}

__global__ void body_range_kernel(const mel_contact* cont, int n, int nb, int* b_cont0)
{
    // b_cont0[b] = first index with bodyS >= b (list is body-major)
    int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b > nb) return;
    int lo = 0, hi = n;
    while (lo < hi) { int mid = (lo + hi) >> 1; if (cont[mid].bodyS < b) lo = mid + 1; else hi = mid; }
    b_cont0[b] = lo;
}

// Newly created elements leave vgapn/vgapt unassigned in the reference: they keep the values of the
// element pushed before them in the slave body's list (the reused new_contact variable,
// Code/Proximity.h:286-313); self contacts use a fresh variable (Code/Proximity.h:350).
__global__ void carry_kernel(const mel_dev d, mel_contact* cont, const int* b_cont0)
{
    int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= d.nb) return;
    double vn = 0., vt = 0.;
    for (int c = b_cont0[b]; c < b_cont0[b + 1]; c++) {
        mel_contact& k = cont[c];
        if (k.bodyM == b) { if (k.pad_) { k.vgapn = 0.; k.vgapt = 0.; } k.pad_ = 0; continue; }
        if (k.pad_) { k.vgapn = vn; k.vgapt = vt; k.pad_ = 0; }
        else { vn = k.vgapn; vt = k.vgapt; }
    }
}

__global__ void inc_range_kernel(const int* inc_task, int ninc, const int* task, const int* slot_off,
                                 const mel_dev d, int2* rng)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= ninc) return;
    int t = inc_task[i];
    int gS = task[4 * t + 1], slot0 = task[4 * t + 3];
    int nS = d.bd_e0[gS + 1] - d.bd_e0[gS];
    rng[i] = make_int2(slot_off[slot0], slot_off[slot0 + nS]);
}

} // namespace mel

// =============================================================================================
// host driver
// =============================================================================================
#include "mel_prox_host.h"

static int ensure(void** p, size_t* cap_bytes, size_t need)
{
    if (need <= *cap_bytes && *p) return 0;
    size_t nc = need + need / 2 + 4096;
    void* np = nullptr;
    if (cudaMalloc(&np, nc) != cudaSuccess) return 1;
    if (*p) cudaFree(*p);
    *p = np;
    *cap_bytes = nc;
    return 0;
}

// Rebuilds b_cont0 and the per-entry index of the current list (d.cont, d.ncont).
int mel_index_contacts(mel_dev& d, mel_prox_state& P, cudaStream_t s)
{
    using namespace mel;
    body_range_kernel<<<(d.nb + 1 + 127) / 128, 128, 0, s>>>(d.cont, d.ncont, d.nb, P.b_cont0);
    cudaMemsetAsync(P.e_cnt, 0, sizeof(int) * (d.ne + 1), s);
    if (d.ncont > 0) entry_count_kernel<<<(d.ncont + 127) / 128, 128, 0, s>>>(d, d.cont, d.ncont, P.e_cnt);
    mel_scan_exclusive(P.e_cnt, P.e_ptr, d.ne, s);
    if (ensure((void**)&P.e_list, &P.e_list_bytes, sizeof(int) * (size_t)(d.ncont + 1))) return MEL_ERR_OOM;
    cudaMemcpyAsync(P.e_cur, P.e_ptr, sizeof(int) * (d.ne + 1), cudaMemcpyDeviceToDevice, s);
    entry_index_kernel<<<(d.nb + 127) / 128, 128, 0, s>>>(d, d.cont, P.b_cont0, P.e_cur, P.e_list);
    return cudaGetLastError() == cudaSuccess ? MEL_OK : MEL_ERR_CUDA;
}

int mel_run_proximity(mel_dev& d, mel_prox_state& P, const mel_prox_host& H, cudaStream_t s)
{
    using namespace mel;
    const int nb = d.nb;
    // 1. border boxes
    aabb_kernel<<<(d.nbd * 32 + 255) / 256, 256, 0, s>>>(d, P.aabb, P.shmin, P.shmax);
    // 2. neighbours (retry with a larger capacity on overflow)
    for (int attempt = 0; attempt < 4; attempt++) {
        cudaMemsetAsync(d.err + MEL_E_NBR_OVERFLOW, 0, sizeof(unsigned), s);
        cudaMemsetAsync(d.err + MEL_E_NBR_NEED, 0, sizeof(unsigned), s);
        neighbour_kernel<<<(nb * 32 + 255) / 256, 256, 0, s>>>(d, P.aabb, P.shmin, P.shmax, P.nbr, P.nbn, P.nbr_cap);
        unsigned ov[2];
        cudaMemcpyAsync(ov, d.err + MEL_E_NBR_OVERFLOW, sizeof(unsigned) * 1, cudaMemcpyDeviceToHost, s);
        cudaMemcpyAsync(ov + 1, d.err + MEL_E_NBR_NEED, sizeof(unsigned), cudaMemcpyDeviceToHost, s);
        if (cudaStreamSynchronize(s) != cudaSuccess) return MEL_ERR_CUDA;
        if (!ov[0]) break;
        int need = (int)ov[1] + 16;
        cudaFree(P.nbr); P.nbr = nullptr;
        if (cudaMalloc(&P.nbr, sizeof(int) * 3 * (size_t)need * nb) != cudaSuccess) return MEL_ERR_OOM;
        P.nbr_cap = need;
    }
    // 3. task list on the host (reference loop order, Code/Proximity.h:207-212 and 346-356)
    P.h_nbn.resize(nb);
    P.h_nbr.resize((size_t)3 * P.nbr_cap * nb);
    cudaMemcpyAsync(P.h_nbn.data(), P.nbn, sizeof(int) * nb, cudaMemcpyDeviceToHost, s);
    cudaMemcpyAsync(P.h_nbr.data(), P.nbr, sizeof(int) * 3 * (size_t)P.nbr_cap * nb, cudaMemcpyDeviceToHost, s);
    if (cudaStreamSynchronize(s) != cudaSuccess) return MEL_ERR_CUDA;
    std::vector<int>& T = P.h_task;
    T.clear();
    std::vector<int> key;            // master body of each task
    int slot = 0;
    for (int b = 0; b < nb; b++) {
        for (int g = H.b_bd0[b]; g < H.b_bd0[b + 1]; g++) {
            int nS = H.bd_e0[g + 1] - H.bd_e0[g];
            for (int q = 0; q < P.h_nbn[b]; q++) {
                T.push_back(b); T.push_back(g); T.push_back(q); T.push_back(slot);
                key.push_back(P.h_nbr[(size_t)3 * P.nbr_cap * b + 3 * q]);
                slot += nS;
            }
        }
        if (d.self_contact && H.b_type[b] == MEL_BODY_DEFORMABLE && !H.b_per[b]) {
            for (int g = H.b_bd0[b]; g < H.b_bd0[b + 1]; g++) {
                int nS = H.bd_e0[g + 1] - H.bd_e0[g];
                T.push_back(b); T.push_back(g); T.push_back(-1); T.push_back(slot);
                key.push_back(b);
                slot += nS;
            }
        }
    }
    int ntask = (int)(T.size() / 4);
    int nslot = slot;
    // incoming task lists: tasks grouped by master body, each group in task order (= send order)
    std::vector<int> inc_cnt(nb + 1, 0);
    for (int t = 0; t < ntask; t++) inc_cnt[key[t] + 1]++;
    for (int b = 0; b < nb; b++) inc_cnt[b + 1] += inc_cnt[b];
    P.h_inc_task.assign(ntask > 0 ? ntask : 1, 0);
    {
        std::vector<int> cur(inc_cnt.begin(), inc_cnt.end() - 1);
        for (int t = 0; t < ntask; t++) P.h_inc_task[cur[key[t]]++] = t;
    }
    if (ensure((void**)&P.task, &P.task_bytes, sizeof(int) * 4 * (size_t)(ntask + 1))) return MEL_ERR_OOM;
    if (ensure((void**)&P.inc_task, &P.inc_task_bytes, sizeof(int) * (size_t)(ntask + 1))) return MEL_ERR_OOM;
    if (ensure((void**)&P.slot_cnt, &P.slot_bytes, sizeof(int) * (size_t)(nslot + 1))) return MEL_ERR_OOM;
    if (ensure((void**)&P.slot_off, &P.slot_off_bytes, sizeof(int) * (size_t)(nslot + 1))) return MEL_ERR_OOM;
    if (ensure((void**)&P.inc_rng, &P.inc_rng_bytes, sizeof(int2) * (size_t)(ntask + 1))) return MEL_ERR_OOM;
    if (ntask > 0) {
        cudaMemcpyAsync(P.task, T.data(), sizeof(int) * 4 * ntask, cudaMemcpyHostToDevice, s);
        cudaMemcpyAsync(P.inc_task, P.h_inc_task.data(), sizeof(int) * ntask, cudaMemcpyHostToDevice, s);
    }
    cudaMemcpyAsync(P.b_inc0, inc_cnt.data(), sizeof(int) * (nb + 1), cudaMemcpyHostToDevice, s);
    // 4. count, scan
    if (ntask > 0) count_kernel<<<(ntask * 32 + 255) / 256, 256, 0, s>>>(d, P.task, ntask, P.nbr, P.nbr_cap, P.slot_cnt);
    mel_scan_exclusive(P.slot_cnt, P.slot_off, nslot, s);
    int total = 0;
    cudaMemcpyAsync(&total, P.slot_off + nslot, sizeof(int), cudaMemcpyDeviceToHost, s);
    if (cudaStreamSynchronize(s) != cudaSuccess) return MEL_ERR_CUDA;
    // 5. write the new list into the spare buffer, inheriting from the current one
    if (ensure((void**)&P.cont_alt, &P.cont_alt_bytes, sizeof(mel_contact) * (size_t)(total + 1))) return MEL_ERR_OOM;
    if (ntask > 0)
        write_kernel<<<(ntask * 32 + 255) / 256, 256, 0, s>>>(d, P.task, ntask, P.nbr, P.nbr_cap, P.slot_off, P.cont_alt,
                                                             d.cont, P.e_ptr, P.e_list, d.ncont > 0 ? 1 : 0);
    // swap buffers
    mel_contact* old = d.cont;
    size_t old_bytes = P.cont_bytes;
    d.cont = P.cont_alt; P.cont_bytes = P.cont_alt_bytes;
    P.cont_alt = old; P.cont_alt_bytes = old_bytes;
    d.ncont = total;
    if (ensure((void**)&P.cont_w, &P.cont_w_bytes, sizeof(double) * (size_t)(total + 1))) return MEL_ERR_OOM;
    cudaMemsetAsync(P.cont_w, 0, sizeof(double) * (total + 1), s);
    d.cont_w = P.cont_w;
    // 6. index structures of the new list
    if (ntask > 0) inc_range_kernel<<<(ntask + 127) / 128, 128, 0, s>>>(P.inc_task, ntask, P.task, P.slot_off, d, P.inc_rng);
    d.inc_rng = P.inc_rng;
    d.b_inc0 = P.b_inc0;
    int rc = mel_index_contacts(d, P, s);
    d.b_cont0 = P.b_cont0;
    carry_kernel<<<(nb + 127) / 128, 128, 0, s>>>(d, d.cont, P.b_cont0);
    P.ntask = ntask; P.nslot = nslot;
    if (rc) return rc;
    return cudaGetLastError() == cudaSuccess ? MEL_OK : MEL_ERR_CUDA;
}

// Index structures for a list supplied by the caller (mel_set_contacts): incoming ranges are built
// on the host from the list itself (contacts grouped by master body, in list order).
int mel_index_external(mel_dev& d, mel_prox_state& P, const mel_contact* host_list, int n, cudaStream_t s)
{
    int nb = d.nb;
    std::vector<int> cnt(nb + 1, 0);
    std::vector<int2> rng;
    std::vector<std::vector<int2>> per(nb);
    for (int i = 0; i < n; ) {
        int j = i;
        while (j < n && host_list[j].bodyS == host_list[i].bodyS && host_list[j].bodyM == host_list[i].bodyM) j++;
        per[host_list[i].bodyM].push_back(make_int2(i, j));
        i = j;
    }
    for (int b = 0; b < nb; b++) { cnt[b + 1] = cnt[b] + (int)per[b].size(); for (auto& r : per[b]) rng.push_back(r); }
    if (ensure((void**)&P.inc_rng, &P.inc_rng_bytes, sizeof(int2) * (rng.size() + 1))) return MEL_ERR_OOM;
    if (!rng.empty()) cudaMemcpyAsync(P.inc_rng, rng.data(), sizeof(int2) * rng.size(), cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync(P.b_inc0, cnt.data(), sizeof(int) * (nb + 1), cudaMemcpyHostToDevice, s);
    d.inc_rng = P.inc_rng;
    d.b_inc0 = P.b_inc0;
    int rc = mel_index_contacts(d, P, s);
    d.b_cont0 = P.b_cont0;
    if (cudaStreamSynchronize(s) != cudaSuccess) return MEL_ERR_CUDA;
    return rc;
}
