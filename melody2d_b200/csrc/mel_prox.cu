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
    bool nonfinite = false;          // the comparisons below pass over NaN, so it is tested apart
    for (int e = d.bd_e0[g] + lane; e < d.bd_e0[g + 1]; e += 32) {
        double2 p = d.x[n0 + d.e_node[e]];
        nonfinite |= !isfinite(p.x) || !isfinite(p.y);
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
    nonfinite = __any_sync(0xffffffffu, nonfinite);
    if (lane == 0) {
        double invperiod = 1. / d.period;
        double f0 = floor((xmin - d.xmin) * invperiod), f1 = floor((xmax - d.xmin) * invperiod);
        // a box that is not finite, or that spans more periods than any body can, comes from a
        // diverged state; it is reported and left out of the neighbour search, whose shift loop
        // it would otherwise drive through billions of iterations
        bool finite = !nonfinite && isfinite(xmin) && isfinite(xmax) && isfinite(ymin) && isfinite(ymax);
        bool sane = finite && fabs(f0) < 1.e6 && fabs(f1) < 1.e6 && f1 - f0 <= MEL_MAX_SHIFT_SPAN;
        if (!sane) {
            atomicOr(&d.err[MEL_E_NAN], finite ? 2u : 1u);
            xmin = 1.e300; xmax = -1.e300; ymin = 1.e300; ymax = -1.e300; f0 = 0.; f1 = -1.;
        }
        aabb[4 * g] = xmin; aabb[4 * g + 1] = xmax; aabb[4 * g + 2] = ymin; aabb[4 * g + 3] = ymax;
        shmin[g] = (int)f0;
        shmax[g] = (int)f1;
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

// ---------------------------------------------------------------------------------------------
// segment blocks: bounding boxes of MEL_SEGB consecutive segments of a border (node1/node2 positions
// with the border's own period shifts).  Used only to skip segments that cannot pass
// Detect_Segment_Proximity; the boxes are widened by the detection distance plus a margin, so the
// accepted candidates and their order are unchanged.
// ---------------------------------------------------------------------------------------------
__global__ void segblock_kernel(mel_dev d)
{
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= d.nblk) return;
    int g = d.blk_border[k];
    int b = d.bd_body[g];
    int e0 = d.bd_e0[g];
    int nseg = d.bd_e0[g + 1] - e0 - 1;
    int s0 = (k - d.bd_blk0[g]) * MEL_SEGB;
    int s1 = min(s0 + MEL_SEGB, nseg);
    int n0 = d.b_node0[b];
    double xmin = 1.e300, xmax = -1.e300, ymin = 1.e300, ymax = -1.e300;
    for (int sg = s0; sg < s1; sg++) {
        int e = e0 + sg;
        for (int j = 1; j <= 2; j++) {
            // shifted (regular search) and unshifted (self search) abscissae both count
            double2 p = d.x[n0 + d.e_sn[4 * e + j]];
            double x = p.x + d.period * d.e_ss[4 * e + j];
            xmin = fmin(xmin, fmin(x, p.x)); xmax = fmax(xmax, fmax(x, p.x));
            ymin = fmin(ymin, p.y); ymax = fmax(ymax, p.y);
        }
    }
    d.seg_blk[k] = make_double4(xmin, xmax, ymin, ymax);
}

// superblock boxes: unions of MEL_SEGB2 consecutive block boxes of one border
__global__ void superblock_kernel(mel_dev d)
{
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= d.nsblk) return;
    int g = d.sblk_border[k];
    int b0 = d.bd_blk0[g] + (k - d.bd_sblk0[g]) * MEL_SEGB2;
    int b1 = min(b0 + MEL_SEGB2, d.bd_blk0[g + 1]);
    double4 u = make_double4(1.e300, -1.e300, 1.e300, -1.e300);
    for (int j = b0; j < b1; j++) {
        double4 bb = d.seg_blk[j];
        u.x = fmin(u.x, bb.x); u.y = fmax(u.y, bb.y); u.z = fmin(u.z, bb.z); u.w = fmax(u.w, bb.w);
    }
    d.seg_sblk[k] = u;
}

__device__ __forceinline__ bool block_may_detect(const double4& bb, double xs, double ys, double m)
{
    return !(xs < bb.x - m || xs > bb.y + m || ys < bb.z - m || ys > bb.w + m);
}

// Calls body(kb) for each block kb (border-local index) of border g whose superblock box and
// block box both lie within `margin` of (x, y), in ascending block order.
template <typename F>
__device__ __forceinline__ void for_near_blocks(const mel_dev& d, int g, double x, double y, double margin, F&& body)
{
    const int blk0 = d.bd_blk0[g], blk1 = d.bd_blk0[g + 1];
    for (int ks = d.bd_sblk0[g]; ks < d.bd_sblk0[g + 1]; ks++) {
        if (!block_may_detect(d.seg_sblk[ks], x, y, margin)) continue;
        const int k0 = blk0 + (ks - d.bd_sblk0[g]) * MEL_SEGB2;
        const int k1 = min(k0 + MEL_SEGB2, blk1);
        for (int k = k0; k < k1; k++)
            if (block_may_detect(d.seg_blk[k], x, y, margin)) body(k - blk0);
    }
}

// regular task: slave node kS of global border gS of body bS against neighbour (bM, rM, shM)
template <typename F>
__device__ __forceinline__ void enum_regular(const mel_dev& d, int bS, int gS, int kS, int bM, int rM, int shM, F&& f)
{
    int gM = d.b_bd0[bM] + rM;
    int eM0 = d.bd_e0[gM], nM = d.bd_e0[gM + 1] - eM0;
    int eS = d.bd_e0[gS] + kS;
    double2 xs = d.x[d.b_node0[bS] + d.e_node[eS]];
    double dd = d.b_dist[3 * bS + 1], cd = d.b_dist[3 * bS + 2];
    double margin = dd * 1.0001 + 1e-12 * (fabs(xs.x) + fabs(xs.y) + fabs(d.period * shM)) + 1e-15;
    double xrel = xs.x - d.period * shM;
    int mb = d.b_node0[bM];
    for_near_blocks(d, gM, xrel, xs.y, margin, [&](int kb) {
        int s0 = kb * MEL_SEGB;
        int s1 = min(s0 + MEL_SEGB, nM - 1);
        for (int seg = s0; seg < s1; seg++) {
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
    });
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
    double margin = dd * 1.0001 + 1e-12 * (fabs(xs.x) + fabs(xs.y)) + 1e-15;
    for (int gM = d.b_bd0[bS]; gM < d.b_bd0[bS + 1]; gM++) {
        int eM0 = d.bd_e0[gM], nM = d.bd_e0[gM + 1] - eM0;
        for_near_blocks(d, gM, xs.x, xs.y, margin, [&](int kb) {
            int s0 = kb * MEL_SEGB;
            int s1 = min(s0 + MEL_SEGB, nM - 1);
            for (int seg = s0; seg < s1; seg++) {
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
        });
    }
}

// ---------------------------------------------------------------------------------------------
// task list on the device.  Task t: slave body, slave border (global), neighbour index q (-1: self),
// slave border nodes; tasks of a body are contiguous: (border, neighbour) pairs in the reference's
// loop order (Code/Proximity.h:207-212), then one self task per border (Code/Proximity.h:346-356).
// ---------------------------------------------------------------------------------------------
__device__ __forceinline__ bool has_self(const mel_dev& d, int b)
{
    return d.self_contact && d.b_type[b] == MEL_BODY_DEFORMABLE && !d.b_per[b];
}

// per body: task count and slot count (slave border nodes summed over its tasks)
__global__ void task_count_kernel(mel_dev d, const int* nbn, int* tcnt, int* scnt)
{
    int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= d.nb) return;
    int nbd = d.b_bd0[b + 1] - d.b_bd0[b];
    int nent = d.bd_e0[d.b_bd0[b + 1]] - d.bd_e0[d.b_bd0[b]];
    int per = nbn[b] + (has_self(d, b) ? 1 : 0);
    tcnt[b] = nbd * per;
    scnt[b] = nent * per;
}

// task t = (slave body, slave border, neighbour q or -1 for self, first slot), its slave border node
// count, its first slot and its master body; inc_cnt counts the tasks of each master body
__global__ void task_fill_kernel(mel_dev d, const int* nbr, const int* nbn, int cap, const int* btask0,
                                 const int* bslot0, int4* task, int* tns, int* tslot, int* tkey, int* inc_cnt)
{
    int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= d.nb) return;
    int t = btask0[b];
    int slot = bslot0[b];
    const int* nb = nbr + (size_t)3 * cap * b;
    for (int g = d.b_bd0[b]; g < d.b_bd0[b + 1]; g++) {
        int nS = d.bd_e0[g + 1] - d.bd_e0[g];
        for (int q = 0; q < nbn[b]; q++) {
            int key = nb[3 * q];
            task[t] = make_int4(b, g, q, slot); tns[t] = nS; tslot[t] = slot; tkey[t] = key;
            atomicAdd(&inc_cnt[key], 1);
            t++; slot += nS;
        }
    }
    if (has_self(d, b))
        for (int g = d.b_bd0[b]; g < d.b_bd0[b + 1]; g++) {
            int nS = d.bd_e0[g + 1] - d.bd_e0[g];
            task[t] = make_int4(b, g, -1, slot); tns[t] = nS; tslot[t] = slot; tkey[t] = b;
            atomicAdd(&inc_cnt[b], 1);
            t++; slot += nS;
        }
}

__global__ void count_kernel(mel_dev d, const int4* task, int ntask, const int* nbr, int cap, int* slot_cnt)
{
    int t = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    int lane = threadIdx.x & 31;
    if (t >= ntask) return;
    int4 tk = task[t];
    int bS = tk.x, gS = tk.y, q = tk.z, slot0 = tk.w;
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

__global__ void write_kernel(mel_dev d, const int4* task, int ntask, const int* nbr, int cap, const int* slot_off,
                             mel_contact* out, const mel_contact* old, const int* old_eptr, const int* old_elist,
                             int have_old)
{
    int t = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    int lane = threadIdx.x & 31;
    if (t >= ntask) return;
    int4 tk = task[t];
    int bS = tk.x, gS = tk.y, q = tk.z, slot0 = tk.w;
    int rS = gS - d.b_bd0[bS];
    int eS0 = d.bd_e0[gS];
    int nS = d.bd_e0[gS + 1] - eS0;
    for (int kS = lane; kS < nS; kS += 32) {
        int pos = slot_off[slot0 + kS];
        const int end = slot_off[slot0 + kS + 1];   // the count pass found end - pos candidates
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
                if (pos < end) out[pos] = c;
                pos++;
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
                if (pos < end) out[pos] = c;
                pos++;
            });
        }
        if (pos != end) atomicOr(&d.err[MEL_E_BOUNDS], 4u);   // count and write passes disagree
    }
}

// ---------------------------------------------------------------------------------------------
// incoming (master-side) contact ranges of each body in send order.  Send_contact_forces runs over
// the sending bodies in index order (Code/Solver.h:61-62) and each sender over its contact list, so
// the incoming ranges of master body B are the tasks whose master is B, in ascending task order.
// Tasks are grouped by master with a counting pass and an atomic fill, then each group is put back
// in ascending order by a rank sort (task ids are unique), one warp per master body.
// ---------------------------------------------------------------------------------------------
__global__ void inc_fill_kernel(const int* tkey, int ntask, int* cur, int* tmp)
{
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= ntask) return;
    tmp[atomicAdd(&cur[tkey[t]], 1)] = t;
}

__global__ void inc_sort_kernel(int nb, const int* inc0, const int* tmp, int* sorted)
{
    int B = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    int lane = threadIdx.x & 31;
    if (B >= nb) return;
    int i0 = inc0[B], n = inc0[B + 1] - i0;
    for (int i = lane; i < n; i += 32) {
        int t = tmp[i0 + i], r = 0;
        for (int j = 0; j < n; j++) r += (tmp[i0 + j] < t);
        sorted[i0 + r] = t;
    }
}

__global__ void inc_range_kernel(const int* sorted, int n, const int* tslot, const int* tns, const int* slot_off, int2* rng)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int t = sorted[i];
    rng[i] = make_int2(slot_off[tslot[t]], slot_off[tslot[t] + tns[t]]);
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

} // namespace mel

// =============================================================================================
// host driver
// =============================================================================================
#include "mel_prox_host.h"

static int ensure_impl(void** p, size_t* cap_bytes, size_t need, const char* what)
{
    if (need <= *cap_bytes && *p) return 0;
    size_t nc = need + need / 2 + 4096;
    void* np = nullptr;
    cudaError_t e = cudaMalloc(&np, nc);
    if (e != cudaSuccess) {
        mel_set_error("allocation of %zu bytes for %s failed: %s", nc, what, cudaGetErrorString(e));
        return 1;
    }
    if (*p) cudaFree(*p);
    *p = np;
    *cap_bytes = nc;
    return 0;
}
#define ensure(p, cap, need) ensure_impl(p, cap, need, #p)

// launch errors and stream failures of the pipeline, reported with their CUDA error and line
static int launch_status(int line)
{
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) return MEL_OK;
    mel_set_cuda_error(e, "proximity kernel launch", __FILE__, line);
    return MEL_ERR_CUDA;
}
static bool sync_failed(cudaStream_t s, int line)
{
    cudaError_t e = cudaStreamSynchronize(s);
    if (e == cudaSuccess) return false;
    mel_set_cuda_error(e, "proximity stream", __FILE__, line);
    return true;
}

// Exclusive scan of n ints into out[0..n] (out[n] = total): a block scan per 1024 entries, the
// block totals scanned the same way, then the block offsets added.  Deterministic; the block
// totals live in the state's persistent scratch (no allocation once it has grown).
static size_t scan_scratch_ints(int n)
{
    size_t t = 0;
    while (true) {
        int nblk = (n + SCAN_BLOCK) / SCAN_BLOCK;
        t += (size_t)nblk + 1 + nblk + 2;
        if (nblk <= 1) break;
        n = nblk;
    }
    return t;
}

static void scan_rec(const int* in, int* out, int n, int* ws, int& launches, cudaStream_t s)
{
    int nblk = (n + SCAN_BLOCK) / SCAN_BLOCK;     // covers index n as well
    int* sums = ws;
    int* soff = ws + nblk + 1;
    mel::scan_block_kernel<<<nblk, SCAN_BLOCK, 0, s>>>(in, out, n, sums);
    launches++;
    if (nblk == 1) return;                        // one block: out[n] already holds the total
    scan_rec(sums, soff, nblk, soff + nblk + 2, launches, s);
    mel::scan_add_kernel<<<nblk, SCAN_BLOCK, 0, s>>>(out, n + 1, soff);
    launches++;
}

int mel_scan_exclusive(const int* in, int* out, int n, mel_prox_state& P, cudaStream_t s)
{
    if (ensure((void**)&P.scan_ws, &P.scan_ws_bytes, sizeof(int) * scan_scratch_ints(n))) return MEL_ERR_OOM;
    scan_rec(in, out, n, P.scan_ws, P.launches, s);
    return MEL_OK;
}

// Rebuilds b_cont0 and the per-entry index of the current list (d.cont, d.ncont).
int mel_index_contacts(mel_dev& d, mel_prox_state& P, cudaStream_t s)
{
    using namespace mel;
    body_range_kernel<<<(d.nb + 1 + 127) / 128, 128, 0, s>>>(d.cont, d.ncont, d.nb, P.b_cont0); P.launches++;
    cudaMemsetAsync(P.e_cnt, 0, sizeof(int) * (d.ne + 1), s);
    if (d.ncont > 0) { entry_count_kernel<<<(d.ncont + 127) / 128, 128, 0, s>>>(d, d.cont, d.ncont, P.e_cnt); P.launches++; }
    if (mel_scan_exclusive(P.e_cnt, P.e_ptr, d.ne, P, s)) return MEL_ERR_OOM;
    if (ensure((void**)&P.e_list, &P.e_list_bytes, sizeof(int) * (size_t)(d.ncont + 1))) return MEL_ERR_OOM;
    cudaMemcpyAsync(P.e_cur, P.e_ptr, sizeof(int) * (d.ne + 1), cudaMemcpyDeviceToDevice, s);
    entry_index_kernel<<<(d.nb + 127) / 128, 128, 0, s>>>(d, d.cont, P.b_cont0, P.e_cur, P.e_list); P.launches++;
    return launch_status(__LINE__);
}

int mel_run_proximity(mel_dev& d, mel_prox_state& P, const mel_prox_host& H, cudaStream_t s)
{
    using namespace mel;
    (void)H;
    const int nb = d.nb;
    // 1. border boxes and segment-block boxes
    aabb_kernel<<<(d.nbd * 32 + 255) / 256, 256, 0, s>>>(d, P.aabb, P.shmin, P.shmax); P.launches++;
    if (d.nblk > 0) { segblock_kernel<<<(d.nblk + 127) / 128, 128, 0, s>>>(d); P.launches++; }
    if (d.nsblk > 0) { superblock_kernel<<<(d.nsblk + 127) / 128, 128, 0, s>>>(d); P.launches++; }
    // 2. neighbours and the task list; one read-back: overflow flag, task count, slot count
    int ntask = 0, nslot = 0;
    bool overflow = true;
    for (int attempt = 0; attempt < 4 && overflow; attempt++) {
        cudaMemsetAsync(d.err + MEL_E_NBR_OVERFLOW, 0, sizeof(unsigned), s);
        cudaMemsetAsync(d.err + MEL_E_NBR_NEED, 0, sizeof(unsigned), s);
        neighbour_kernel<<<(nb * 32 + 255) / 256, 256, 0, s>>>(d, P.aabb, P.shmin, P.shmax, P.nbr, P.nbn, P.nbr_cap); P.launches++;
        task_count_kernel<<<(nb + 127) / 128, 128, 0, s>>>(d, P.nbn, P.tcnt, P.scnt); P.launches++;
        if (mel_scan_exclusive(P.tcnt, P.btask0, nb, P, s)) return MEL_ERR_OOM;
        if (mel_scan_exclusive(P.scnt, P.bslot0, nb, P, s)) return MEL_ERR_OOM;
        unsigned hv[MEL_E_NWORDS];
        cudaMemcpyAsync(hv, d.err, sizeof hv, cudaMemcpyDeviceToHost, s);
        cudaMemcpyAsync(&ntask, P.btask0 + nb, sizeof(int), cudaMemcpyDeviceToHost, s);
        cudaMemcpyAsync(&nslot, P.bslot0 + nb, sizeof(int), cudaMemcpyDeviceToHost, s);
        if (sync_failed(s, __LINE__)) return MEL_ERR_CUDA;
        if (hv[MEL_E_NAN]) {
            mel_set_error(hv[MEL_E_NAN] & 1u ? "non-finite node positions at the proximity update"
                                             : "a border box spans more than %d periods: diverged positions",
                          MEL_MAX_SHIFT_SPAN);
            return MEL_ERR_NAN;
        }
        hv[0] = hv[MEL_E_NBR_OVERFLOW]; hv[1] = hv[MEL_E_NBR_NEED];
        overflow = hv[0] != 0;
        if (!overflow) break;
        int need = (int)hv[1] + 16;
        cudaFree(P.nbr); P.nbr = nullptr;
        if (cudaMalloc(&P.nbr, sizeof(int) * 3 * (size_t)need * nb) != cudaSuccess) {
            mel_set_error("allocation of neighbour lists (%d per body) failed", need);
            return MEL_ERR_OOM;
        }
        P.nbr_cap = need;
    }
    if (overflow) { mel_set_error("neighbour lists still over capacity after 4 attempts"); return MEL_ERR_BOUNDS; }
    if (ensure((void**)&P.task, &P.task_bytes, sizeof(int4) * (size_t)(ntask + 1))) return MEL_ERR_OOM;
    if (ensure((void**)&P.tns, &P.tns_bytes, sizeof(int) * (size_t)(ntask + 1))) return MEL_ERR_OOM;
    if (ensure((void**)&P.tslot, &P.tslot_bytes, sizeof(int) * (size_t)(ntask + 1))) return MEL_ERR_OOM;
    if (ensure((void**)&P.tkey, &P.tkey_bytes, sizeof(int) * (size_t)(ntask + 1))) return MEL_ERR_OOM;
    if (ensure((void**)&P.inc_task, &P.inc_task_bytes, sizeof(int) * 2 * (size_t)(ntask + 1))) return MEL_ERR_OOM;
    int4* task = (int4*)P.task;
    cudaMemsetAsync(P.tcnt, 0, sizeof(int) * (nb + 1), s);
    if (ntask > 0) {
        task_fill_kernel<<<(nb + 127) / 128, 128, 0, s>>>(d, P.nbr, P.nbn, P.nbr_cap, P.btask0, P.bslot0, task, P.tns,
                                                          P.tslot, P.tkey, P.tcnt);
        P.launches++;
    }
    if (ensure((void**)&P.slot_cnt, &P.slot_bytes, sizeof(int) * (size_t)(nslot + 1))) return MEL_ERR_OOM;
    if (ensure((void**)&P.slot_off, &P.slot_off_bytes, sizeof(int) * (size_t)(nslot + 1))) return MEL_ERR_OOM;
    // 3. count, scan, total
    if (ntask > 0) { count_kernel<<<(ntask * 32 + 255) / 256, 256, 0, s>>>(d, task, ntask, P.nbr, P.nbr_cap, P.slot_cnt); P.launches++; }
    if (mel_scan_exclusive(P.slot_cnt, P.slot_off, nslot, P, s)) return MEL_ERR_OOM;
    int total = 0;
    cudaMemcpyAsync(&total, P.slot_off + nslot, sizeof(int), cudaMemcpyDeviceToHost, s);
    if (sync_failed(s, __LINE__)) return MEL_ERR_CUDA;
    // 4. write the new list into the spare buffer, inheriting from the current one
    if (ensure((void**)&P.cont_alt, &P.cont_alt_bytes, sizeof(mel_contact) * (size_t)(total + 1))) return MEL_ERR_OOM;
    if (ntask > 0) {
        write_kernel<<<(ntask * 32 + 255) / 256, 256, 0, s>>>(d, task, ntask, P.nbr, P.nbr_cap, P.slot_off, P.cont_alt,
                                                             d.cont, P.e_ptr, P.e_list, d.ncont > 0 ? 1 : 0);
        P.launches++;
    }
    mel_contact* old = d.cont;
    size_t old_bytes = P.cont_bytes;
    d.cont = P.cont_alt; P.cont_bytes = P.cont_alt_bytes;
    P.cont_alt = old; P.cont_alt_bytes = old_bytes;
    d.ncont = total;
    if (ensure((void**)&P.cont_w, &P.cont_w_bytes, sizeof(double) * (size_t)(total + 1))) return MEL_ERR_OOM;
    cudaMemsetAsync(P.cont_w, 0, sizeof(double) * (total + 1), s);
    d.cont_w = P.cont_w;
    if (ensure((void**)&P.cont_rt, &P.cont_rt_bytes, 6 * sizeof(double) * (size_t)(total + 1))) return MEL_ERR_OOM;
    d.cont_rt = P.cont_rt;
    // 5. incoming ranges in send order
    if (ensure((void**)&P.inc_rng, &P.inc_rng_bytes, sizeof(int2) * (size_t)(ntask + 1))) return MEL_ERR_OOM;
    if (mel_scan_exclusive(P.tcnt, P.b_inc0, nb, P, s)) return MEL_ERR_OOM;
    if (ntask > 0) {
        int* tmp = P.inc_task;
        int* sorted = P.inc_task + ntask;
        cudaMemcpyAsync(P.tcnt, P.b_inc0, sizeof(int) * nb, cudaMemcpyDeviceToDevice, s);
        inc_fill_kernel<<<(ntask + 127) / 128, 128, 0, s>>>(P.tkey, ntask, P.tcnt, tmp); P.launches++;
        inc_sort_kernel<<<(nb * 32 + 255) / 256, 256, 0, s>>>(nb, P.b_inc0, tmp, sorted); P.launches++;
        inc_range_kernel<<<(ntask + 127) / 128, 128, 0, s>>>(sorted, ntask, P.tslot, P.tns, P.slot_off, P.inc_rng); P.launches++;
    }
    d.inc_rng = P.inc_rng;
    d.b_inc0 = P.b_inc0;
    // 6. per-entry index of the new list; vgapn/vgapt carry of new elements
    int rc = mel_index_contacts(d, P, s);
    d.b_cont0 = P.b_cont0;
    carry_kernel<<<(nb + 127) / 128, 128, 0, s>>>(d, d.cont, P.b_cont0); P.launches++;
    P.ntask = ntask; P.nslot = nslot;
    if (rc) return rc;
    return launch_status(__LINE__);
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
    if (sync_failed(s, __LINE__)) return MEL_ERR_CUDA;
    return rc;
}
