// Update_proximity (Code/Proximity.h:48-473) on the device, for one model or for several models
// (the members of a batch) with the same launches.
//
// Stages (all integer bookkeeping deterministic, geometry bit-identical to the reference):
//   aabb_kernel        border boxes inflated by the detection distance and their period shifts
//                      (Code/Proximity.h:63-109), one warp per border; segment-block and
//                      superblock boxes for pruning
//   neighbour_kernel   all-pairs (body, border) overlap with periodic shifts and de-duplication
//                      (Code/Proximity.h:112-169), one warp per body, lanes over candidate bodies
//   task_count / scan / task_fill   task list: one task per (slave body, slave border, neighbour)
//                      in the reference's loop order, then one self task per (slave body, border);
//                      a slot per (task, slave border node)
//   [host read-back]   task and slot totals of every member
//   count_kernel       accepted candidates per slot, one thread per slot (slot_task_kernel maps
//                      slots to tasks)
//   scan               slot offsets = the canonical position of every new contact element; the
//                      slots with candidates are listed for the write pass
//   [host read-back]   contact totals of every member
//   write_kernel       writes the new list in the reference's order; history inheritance searches
//                      the previous list of the same slave border node (Code/Proximity.h:269-284)
//   incoming ranges, entry index, vgap carry   index structures for the next step and update
// Every kernel reads a table of member jobs (mel_prox_job); the host driver is at the end.
#include <cstdio>
#include <cstring>
#include <utility>
#include <vector>
#include <algorithm>
#include "mel_internal.h"
#include "mel_geometry.cuh"
#include "mel_prox_host.h"

struct mel_scan_job { const int* in; int* out; int n; int* sums; };

namespace mel {

// ---------------------------------------------------------------------------------------------
// exclusive scans of int arrays, several per launch (three-phase, deterministic).  Job j scans
// in[0..n) into out[0..n] (out[n] = total); blocks [bpre[j], bpre[j+1]) of a launch serve job j.
// ---------------------------------------------------------------------------------------------
#define SCAN_BLOCK 1024
__device__ __forceinline__ int block_job(const int* bpre, int nj)
{
    int lo = 0, hi = nj;                  // largest j with bpre[j] <= blockIdx.x
    while (hi - lo > 1) { int mid = (lo + hi) >> 1; if (bpre[mid] <= (int)blockIdx.x) lo = mid; else hi = mid; }
    return lo;
}

__global__ void __launch_bounds__(SCAN_BLOCK) scan_block_kernel(const mel_scan_job* J, const int* bpre, int nj)
{
    __shared__ int s[SCAN_BLOCK];
    const int j = block_job(bpre, nj);
    const int* in = J[j].in;
    int* out = J[j].out;
    const int n = J[j].n;
    const int lb = blockIdx.x - bpre[j];
    int i = lb * SCAN_BLOCK + threadIdx.x;
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
    if (threadIdx.x == SCAN_BLOCK - 1) J[j].sums[lb] = s[threadIdx.x];
}
// adds the scanned block totals (in) to out[0..n) block by block
__global__ void __launch_bounds__(SCAN_BLOCK) scan_add_kernel(const mel_scan_job* J, const int* bpre, int nj)
{
    const int j = block_job(bpre, nj);
    const int lb = blockIdx.x - bpre[j];
    int i = lb * SCAN_BLOCK + threadIdx.x;
    if (i < J[j].n) J[j].out[i] += J[j].in[lb];
}

} // namespace mel

namespace mel {

// ---------------------------------------------------------------------------------------------
__device__ __forceinline__ void aabb_item(const mel_dev& d, double* aabb, int* shmin, int* shmax, int g, int lane)
{
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

// the neighbour entries of border g1 (of body b1) against every active body, appended to out at
// `count` in the reference's order (body, border, shift ascending; Code/Proximity.h:112-169): an
// entry already listed for an earlier border of b1 (out[0..count_before)) is not repeated
__device__ __forceinline__ void nbr_scan_all(const mel_dev& d, const double* aabb, const int* shmin, const int* shmax,
                                             int* out, int cap, int b1, int g1, int count_before, int& count, int lane)
{
    const double xmin1 = aabb[4 * g1], xmax1 = aabb[4 * g1 + 1], ymin1 = aabb[4 * g1 + 2], ymax1 = aabb[4 * g1 + 3];
    const int smin1 = shmin[g1], smax1 = shmax[g1];
    const int first_border = (g1 == d.b_bd0[b1]);
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

// neighbour lists by all pairs of bodies, one warp per body
__device__ __forceinline__ void neighbour_item(const mel_dev& d, const double* aabb, const int* shmin, const int* shmax,
                                               int* nbr, int* nbn, int cap, int b1, int lane)
{
    if (b1 >= d.nb) return;
    if (d.b_status[b1] == MEL_STATUS_INACTIVE) { if (lane == 0) nbn[b1] = 0; return; }
    int* out = nbr + (size_t)3 * cap * b1;
    int count = 0;
    for (int g1 = d.b_bd0[b1]; g1 < d.b_bd0[b1 + 1]; g1++) {
        const int count_before = count;   // entries of earlier border1 iterations (dedup scope)
        nbr_scan_all(d, aabb, shmin, shmax, out, cap, b1, g1, count_before, count, lane);
    }
    if (lane == 0) {
        nbn[b1] = count;
        if (count > cap) { atomicOr(&d.err[MEL_E_NBR_OVERFLOW], 1u); atomicMax(&d.err[MEL_E_NBR_NEED], (unsigned)count); }
    }
}

// ---------------------------------------------------------------------------------------------
// cell-list broad phase: the same neighbour lists from a hashed uniform grid.  Each border box is
// binned by its lower corner (x wrapped over the period, so that shifted copies share columns)
// into cells of side cl_h (the largest initial box, widened; columns cl_hx = period / cl_ncx), the
// borders are counting-sorted by bucket, and each border of a body gathers the borders whose
// lower corner lies in a cell that a box of the run's largest width and height overlapping it
// can occupy.  The gathered borders (hash collisions and repeated columns included) are sorted,
// made unique and emitted with the exact overlap and shift tests of the all-pairs pass, so the
// lists are entry for entry those of nbr_scan_all; a border whose cell range or candidate count
// is too large takes the all-pairs pass instead.  A big box is itself a query like any other: the
// borders it can meet have their corners in the cells its extent (widened by the binned boxes'
// largest width and height) covers, or are big themselves.
// ---------------------------------------------------------------------------------------------
#define PROX_THREADS_CL 256  // threads of the job kernels (PROX_THREADS below)
#define CL_CAND 256          // gathered candidates per border (beyond: all-pairs for that border)
#define CL_MAX_CELLS 4096    // cells one border's query visits (beyond: all-pairs)

__device__ __forceinline__ int cl_bucket(const mel_prox_job& j, double x, double y)
{
    // (a coordinate beyond the integer range saturates: such a box is only ever found by the
    // all-pairs pass of the borders that query it)
    long long cx = (long long)floor((x - j.d.xmin) / j.cl_hx);
    long long cw = cx % j.cl_ncx;
    if (cw < 0) cw += j.cl_ncx;
    const long long cy = (long long)floor(y / j.cl_h);
    const unsigned k = (unsigned)cw * 73856093u ^ (unsigned)cy * 19349663u;
    return (int)(k & (unsigned)(j.cl_T - 1));
}

__device__ __forceinline__ bool cl_box_ok(const mel_dev& d, const double* a, int g)
{
    return d.b_status[d.bd_body[g]] != MEL_STATUS_INACTIVE && a[4 * g] <= a[4 * g + 1] && a[4 * g + 2] <= a[4 * g + 3];
}

// a box wider or higher than a cell (a long wall, a plate) is kept out of the grid: every query
// tests it, and its own border takes the all-pairs pass
__device__ __forceinline__ bool cl_big(const mel_prox_job& j, const double* a)
{
    return a[1] - a[0] > j.cl_h || a[3] - a[2] > j.cl_h;
}

// bucket counts and the largest width and height of the binned boxes (non-negative doubles order
// as their bits); big boxes are listed at the end of cl_idx, counted in cl_cur[cl_T]
__device__ __forceinline__ void cl_count_item(const mel_prox_job& j, int g)
{
    const mel_dev& d = j.d;
    if (g >= d.nbd || !cl_box_ok(d, j.aabb, g)) return;
    const double* a = j.aabb + 4 * g;
    if (cl_big(j, a)) { j.cl_idx[d.nbd - 1 - atomicAdd(&j.cl_cur[j.cl_T], 1)] = g; return; }
    atomicMax(&j.cl_w[0], (unsigned long long)__double_as_longlong(a[1] - a[0]));
    atomicMax(&j.cl_w[1], (unsigned long long)__double_as_longlong(a[3] - a[2]));
    atomicAdd(&j.cl_cnt[cl_bucket(j, a[0], a[2])], 1);
}

__device__ __forceinline__ void cl_fill_item(const mel_prox_job& j, int g)
{
    const mel_dev& d = j.d;
    if (g >= d.nbd || !cl_box_ok(d, j.aabb, g)) return;
    const double* a = j.aabb + 4 * g;
    if (cl_big(j, a)) return;
    const int bk = cl_bucket(j, a[0], a[2]);
    j.cl_idx[j.cl_start[bk] + atomicAdd(&j.cl_cur[bk], 1)] = g;
}

__device__ __forceinline__ void cl_zero_item(const mel_prox_job& j, int i)
{
    if (i > j.cl_T) return;
    j.cl_cnt[i] = 0;
    j.cl_cur[i] = 0;
    if (i == 0) { j.cl_w[0] = 0ull; j.cl_w[1] = 0ull; }
}

__device__ __forceinline__ void cl_neighbour_item(const mel_prox_job& j, int b1, int lane)
{
    __shared__ int s_cl[PROX_THREADS_CL / 32][2 * CL_CAND];
    const mel_dev& d = j.d;
    if (b1 >= d.nb) return;
    if (d.b_status[b1] == MEL_STATUS_INACTIVE) { if (lane == 0) j.nbn[b1] = 0; return; }
    int* cand = s_cl[(threadIdx.x >> 5) % (PROX_THREADS_CL / 32)];
    int* srt = cand + CL_CAND;
    const double* aabb = j.aabb;
    const int cap = j.nbr_cap;
    int* out = j.nbr + (size_t)3 * cap * b1;
    const double W = __longlong_as_double((long long)j.cl_w[0]), H = __longlong_as_double((long long)j.cl_w[1]);
    int count = 0;
    for (int g1 = d.b_bd0[b1]; g1 < d.b_bd0[b1 + 1]; g1++) {
        const int count_before = count;
        const double xmin1 = aabb[4 * g1], xmax1 = aabb[4 * g1 + 1], ymin1 = aabb[4 * g1 + 2], ymax1 = aabb[4 * g1 + 3];
        // boxes left out and boxes too far out for integer cell indices: all pairs.  A big box (a
        // wall) queries the cells its own extent covers, which may be many
        bool all = !(xmin1 <= xmax1) || !(ymin1 <= ymax1) ||
                   !(fabs(ymin1 - H) < 1e12 * j.cl_h && fabs(ymax1) < 1e12 * j.cl_h &&
                     fabs(xmin1 - W - d.xmin) < 1e12 * j.cl_hx && fabs(xmax1 - d.xmin) < 1e12 * j.cl_hx);
        long long cx0 = 0, cx1 = -1, cy0 = 0, cy1 = -1;
        if (!all) {
            // a border g2 overlapping g1 (with some shift) has its lower corner in x within
            // [xmin1 - W, xmax1] modulo the period and in y within [ymin1 - H, ymax1]
            cx0 = (long long)floor((xmin1 - W - d.xmin) / j.cl_hx);
            cx1 = (long long)floor((xmax1 - d.xmin) / j.cl_hx);
            cy0 = (long long)floor((ymin1 - H) / j.cl_h);
            cy1 = (long long)floor(ymax1 / j.cl_h);
            // one more cell on every side: a corner's cell is computed from its unshifted position,
            // and rounding may put it across a cell edge from the shifted value tested here
            cx0--; cx1++; cy0--; cy1++;
            if (cx1 - cx0 + 1 > j.cl_ncx) cx1 = cx0 + j.cl_ncx - 1;      // every wrapped column once
            all = cx1 - cx0 + 1 > CL_MAX_CELLS || cy1 - cy0 + 1 > CL_MAX_CELLS ||
                  (cx1 - cx0 + 1) * (cy1 - cy0 + 1) > CL_MAX_CELLS;      // each factor bounded first: no overflow
        }
        int n = 0;
        if (!all) {
            // the cells' bucket ranges looked up by the lanes together (one cell per lane), then
            // their entries taken as one concatenated list, 32 at a time; the owner cell of list
            // item t is found by a search over the per-lane offsets kept in shared memory
            const int ncx = (int)(cx1 - cx0 + 1), ncell = ncx * (int)(cy1 - cy0 + 1);
            int* c_off = srt;                 // [33]: list offset of each lane's cell, then the total
            int* c_e0 = srt + 64;             // [32]: first entry of each lane's cell
            for (int cb = 0; cb < ncell; cb += 32) {
                const int c = cb + lane;
                int e0 = 0, len = 0;
                if (c < ncell) {
                    const long long cx = cx0 + c % ncx, cy = cy0 + c / ncx;
                    const double xc = d.xmin + ((double)cx + 0.5) * j.cl_hx, yc = ((double)cy + 0.5) * j.cl_h;
                    const int bk = cl_bucket(j, xc, yc);
                    e0 = j.cl_start[bk];
                    len = j.cl_start[bk + 1] - e0;
                }
                int incl = len;
                for (int o = 1; o < 32; o <<= 1) {
                    const int t = __shfl_up_sync(0xffffffffu, incl, o);
                    if (lane >= o) incl += t;
                }
                const int total = __shfl_sync(0xffffffffu, incl, 31);
                c_off[lane] = incl - len;
                c_e0[lane] = e0;
                if (lane == 31) c_off[32] = total;
                __syncwarp();
                for (int tb = 0; tb < total; tb += 32) {
                    const int t = tb + lane;
                    bool ok = false;
                    int g2 = -1;
                    if (t < total) {
                        int lo = 0, hi = 32;          // last lane whose offset is <= t
                        while (hi - lo > 1) { const int mid = (lo + hi) >> 1; if (c_off[mid] <= t) lo = mid; else hi = mid; }
                        g2 = j.cl_idx[c_e0[lo] + (t - c_off[lo])];
                        ok = d.bd_body[g2] != b1 && !((aabb[4 * g2 + 3] < ymin1) || (ymax1 < aabb[4 * g2 + 2]));
                    }
                    const unsigned m = __ballot_sync(0xffffffffu, ok);
                    const int pos = n + __popc(m & ((1u << lane) - 1u));
                    if (ok && pos < CL_CAND) cand[pos] = g2;
                    n += __popc(m);
                }
                __syncwarp();
            }
            // the big boxes, outside the grid
            const int nbig = j.cl_cur[j.cl_T];
            for (int e = 0; e < nbig; e += 32) {
                bool ok = false;
                int g2 = -1;
                if (e + lane < nbig) {
                    g2 = j.cl_idx[d.nbd - 1 - (e + lane)];
                    ok = d.bd_body[g2] != b1 && !((aabb[4 * g2 + 3] < ymin1) || (ymax1 < aabb[4 * g2 + 2]));
                }
                const unsigned m = __ballot_sync(0xffffffffu, ok);
                const int pos = n + __popc(m & ((1u << lane) - 1u));
                if (ok && pos < CL_CAND) cand[pos] = g2;
                n += __popc(m);
            }
            all = n > CL_CAND;
        }
        __syncwarp();
        if (all) { nbr_scan_all(d, aabb, j.shmin, j.shmax, out, cap, b1, g1, count_before, count, lane); continue; }
        // stable rank sort of the gathered borders, then the first of each run of equal values
        for (int i = lane; i < n; i += 32) {
            const int v = cand[i];
            int r = 0;
            for (int k = 0; k < n; k++) r += (cand[k] < v) || (cand[k] == v && k < i);
            srt[r] = v;
        }
        __syncwarp();
        const int smin1 = j.shmin[g1], smax1 = j.shmax[g1];
        const int first_border = (g1 == d.b_bd0[b1]);
        for (int base = 0; base < n; base += 32) {
            const int i = base + lane;
            const bool valid = i < n && (i == 0 || srt[i] != srt[i - 1]);
            const int g2 = valid ? srt[i] : 0;
            const int b2 = valid ? d.bd_body[g2] : 0;
            const int r2 = g2 - (valid ? d.b_bd0[b2] : 0);
            int mine = 0;
            for (int pass = 0; pass < 2; pass++) {
                int k = 0;
                if (valid) {
                    const double xmin2 = aabb[4 * g2], xmax2 = aabb[4 * g2 + 1];
                    for (int s = smin1 - j.shmax[g2]; s <= smax1 - j.shmin[g2]; s++) {
                        if ((xmax2 + s * d.period > xmin1) && (xmin2 + s * d.period < xmax1)) {
                            bool dup = false;
                            if (!first_border)
                                for (int q = 0; q < count_before && q < cap; q++)
                                    if (out[3 * q] == b2 && out[3 * q + 1] == r2 && out[3 * q + 2] == s) { dup = true; break; }
                            if (dup) continue;
                            if (pass == 1) {
                                const int pos = mine + k;
                                if (pos < cap) { out[3 * pos] = b2; out[3 * pos + 1] = r2; out[3 * pos + 2] = s; }
                            }
                            k++;
                        }
                    }
                }
                if (pass == 0) {
                    int incl = k;
                    for (int o = 1; o < 32; o <<= 1) {
                        const int t = __shfl_up_sync(0xffffffffu, incl, o);
                        if (lane >= o) incl += t;
                    }
                    const int total = __shfl_sync(0xffffffffu, incl, 31);
                    mine = count + incl - k;
                    count += total;
                }
            }
            __syncwarp();
        }
        __syncwarp();
    }
    if (lane == 0) {
        j.nbn[b1] = count;
        if (count > cap) { atomicOr(&d.err[MEL_E_NBR_OVERFLOW], 1u); atomicMax(&d.err[MEL_E_NBR_NEED], (unsigned)count); }
    }
}

// ---------------------------------------------------------------------------------------------
// segment blocks: bounding boxes of MEL_SEGB consecutive segments of a border (node1/node2 positions
// with the border's own period shifts).  Used only to skip segments that cannot pass
// Detect_Segment_Proximity; the boxes are widened by the detection distance plus a margin, so the
// accepted candidates and their order are unchanged.
// ---------------------------------------------------------------------------------------------
__device__ __forceinline__ void segblock_item(const mel_dev& d, int k)
{
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
__device__ __forceinline__ void superblock_item(const mel_dev& d, int k)
{
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
__device__ __forceinline__ void task_count_item(const mel_dev& d, const int* nbn, int* tcnt, int* scnt, int b)
{
    if (b >= d.nb) return;
    int nbd = d.b_bd0[b + 1] - d.b_bd0[b];
    int nent = d.bd_e0[d.b_bd0[b + 1]] - d.bd_e0[d.b_bd0[b]];
    int per = nbn[b] + (has_self(d, b) ? 1 : 0);
    tcnt[b] = nbd * per;
    scnt[b] = nent * per;
}

// task t = (slave body, slave border, neighbour q or -1 for self, first slot), its slave border node
// count, its first slot and its master body; inc_cnt counts the tasks of each master body
__device__ __forceinline__ void task_fill_item(const mel_dev& d, const int* nbr, const int* nbn, int cap, const int* btask0,
                                               const int* bslot0, int4* task, int* tns, int* tslot, int* tkey, int* inc_cnt,
                                               int b)
{
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

// slot -> task map: warp per task, lanes over its slots
__device__ __forceinline__ void slot_task_item(const mel_dev& d, const int4* task, int ntask, int* tmap, int t, int lane)
{
    if (t >= ntask) return;
    const int4 tk = task[t];
    const int nS = d.bd_e0[tk.y + 1] - d.bd_e0[tk.y];
    for (int kS = lane; kS < nS; kS += 32) tmap[tk.w + kS] = t;
}

// candidates of slot s (one slave border node of one task); one thread per slot, so a task with a
// long slave border (a plate or a wall) spreads over many warps
__device__ __forceinline__ void count_item(const mel_dev& d, const int4* task, const int* tmap, int nslot, const int* nbr,
                                           int cap, int* slot_cnt, int s)
{
    if (s >= nslot) return;
    int t = tmap[s];
    int4 tk = task[t];
    int bS = tk.x, gS = tk.y, q = tk.z, slot0 = tk.w;
    {
        const int kS = s - slot0;
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

// writes the candidates of slot s at their canonical positions; one thread per slot
__device__ __forceinline__ void write_item(const mel_dev& d, const int4* task, const int* tmap, const int* nzlist,
                                           int nnz, const int* nbr, int cap, const int* slot_off, mel_contact* out,
                                           const mel_contact* old, const int* old_eptr, const int* old_elist,
                                           int have_old, int i)
{
    if (i >= nnz) return;
    const int s = nzlist[i];                 // slots with at least one candidate
    int t = tmap[s];
    int4 tk = task[t];
    int bS = tk.x, gS = tk.y, q = tk.z, slot0 = tk.w;
    int rS = gS - d.b_bd0[bS];
    int eS0 = d.bd_e0[gS];
    {
        const int kS = s - slot0;
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
__device__ __forceinline__ void inc_fill_item(const int* tkey, int ntask, int* cur, int* tmp, int t)
{
    if (t >= ntask) return;
    tmp[atomicAdd(&cur[tkey[t]], 1)] = t;
}

__device__ __forceinline__ void inc_sort_item(int nb, const int* inc0, const int* tmp, int* sorted, int B, int lane)
{
    if (B >= nb) return;
    int i0 = inc0[B], n = inc0[B + 1] - i0;
    for (int i = lane; i < n; i += 32) {
        int t = tmp[i0 + i], r = 0;
        for (int j = 0; j < n; j++) r += (tmp[i0 + j] < t);
        sorted[i0 + r] = t;
    }
}

__device__ __forceinline__ void inc_range_item(const int* sorted, int n, const int* tslot, const int* tns,
                                               const int* slot_off, int2* rng, int i)
{
    if (i >= n) return;
    int t = sorted[i];
    rng[i] = make_int2(slot_off[tslot[t]], slot_off[tslot[t] + tns[t]]);
}


// per-body counting sort of a body-major contact list by slave border entry: one warp per body,
// 32 contacts at a time in list order; lanes with the same entry take consecutive places in lane
// order, so every entry lists its contacts in list order (as a serial pass would)
__device__ __forceinline__ void entry_index_item(const mel_dev& d, const mel_contact* cont, const int* b_cont0,
                                                 int* eptr_cnt, int* elist, int b, int lane)
{
    if (b >= d.nb) return;
    const int e_lo = d.bd_e0[d.b_bd0[b]], e_hi = d.bd_e0[d.b_bd0[b + 1]];
    const int c0 = b_cont0[b], c1 = b_cont0[b + 1];
    // eptr_cnt holds the exclusive offsets of this body's entries (prepared by the caller) and is
    // advanced as a cursor; only this warp touches the entries of body b
    for (int base = c0; base < c1; base += 32) {
        const int c = base + lane;
        int e = -1;
        if (c < c1) {
            e = d.bd_e0[d.b_bd0[b] + cont[c].borderS] + cont[c].border_nodeS;
            if (e < e_lo || e >= e_hi) { atomicOr(&d.err[MEL_E_BOUNDS], 2u); e = -1; }
        }
        const unsigned same = __match_any_sync(0xffffffffu, e);
        const int leader = __ffs(same) - 1;
        int pos = 0;
        if (lane == leader && e >= 0) { pos = eptr_cnt[e]; eptr_cnt[e] = pos + __popc(same); }
        pos = __shfl_sync(0xffffffffu, pos, leader) + __popc(same & ((1u << lane) - 1u));
        if (e >= 0) elist[pos] = c;
        __syncwarp();
    }
}

__device__ __forceinline__ void entry_count_item(const mel_dev& d, const mel_contact* cont, int n, int* cnt, int c)
{
    if (c >= n) return;
    int b = cont[c].bodyS;
    int e = d.bd_e0[d.b_bd0[b] + cont[c].borderS] + cont[c].border_nodeS;
    atomicAdd(&cnt[e], 1);
}

__device__ __forceinline__ void body_range_item(const mel_contact* cont, int n, int nb, int* b_cont0, int b)
{
    // b_cont0[b] = first index with bodyS >= b (list is body-major)
    if (b > nb) return;
    int lo = 0, hi = n;
    while (lo < hi) { int mid = (lo + hi) >> 1; if (cont[mid].bodyS < b) lo = mid + 1; else hi = mid; }
    b_cont0[b] = lo;
}

// Newly created elements leave vgapn/vgapt unassigned in the reference: they keep the values of the
// element pushed before them in the slave body's list (the reused new_contact variable,
// Code/Proximity.h:286-313); self contacts use a fresh variable (Code/Proximity.h:350).  One warp
// per body, 32 contacts at a time: a new element takes the values of the last inherited non-self
// element before it (found by ballot within the 32, else carried over from earlier ones).
__device__ __forceinline__ void carry_item(const mel_dev& d, mel_contact* cont, const int* b_cont0, int b, int lane)
{
    if (b >= d.nb) return;
    double vn = 0., vt = 0.;                 // carried value (equal in all lanes)
    const int c0 = b_cont0[b], c1 = b_cont0[b + 1];
    for (int base = c0; base < c1; base += 32) {
        const int c = base + lane;
        const bool valid = c < c1;
        int bodyM = -1, pad = 0;
        double gn = 0., gt = 0.;
        if (valid) { bodyM = cont[c].bodyM; pad = cont[c].pad_; gn = cont[c].vgapn; gt = cont[c].vgapt; }
        const bool self = bodyM == b;
        const bool src = valid && !self && !pad;          // inherited non-self elements set the value
        const unsigned m = __ballot_sync(0xffffffffu, src);
        const unsigned lower = m & ((1u << lane) - 1u);
        const int from = lower ? 31 - __clz(lower) : 0;
        const double sn = __shfl_sync(0xffffffffu, gn, from), st = __shfl_sync(0xffffffffu, gt, from);
        if (valid && pad) {
            if (self) { cont[c].vgapn = 0.; cont[c].vgapt = 0.; }
            else if (lower) { cont[c].vgapn = sn; cont[c].vgapt = st; }
            else { cont[c].vgapn = vn; cont[c].vgapt = vt; }
            cont[c].pad_ = 0;
        } else if (valid && self) {
            cont[c].pad_ = 0;
        }
        if (m) {
            const int last = 31 - __clz(m);
            vn = __shfl_sync(0xffffffffu, gn, last);
            vt = __shfl_sync(0xffffffffu, gt, last);
        }
    }
}

// ---------------------------------------------------------------------------------------------
// job-table launches: blocks [bpre[j], bpre[j+1]) serve member j.  The block copies the member's
// job into shared memory; item `it` of the member is handled by TPI consecutive threads (TPI 32:
// one warp per item, TPI 1: one thread).
// ---------------------------------------------------------------------------------------------
#define PROX_THREADS 256
static_assert(PROX_THREADS == PROX_THREADS_CL, "cell-list scratch is sized for the job kernels' block");
#define JOB_KERNEL(name, TPI, ...)                                                                  \
    __global__ void __launch_bounds__(PROX_THREADS) name(const mel_prox_job* J, const int* bpre, int nj) \
    {                                                                                               \
        __shared__ mel_prox_job sj;                                                                 \
        const int jj = block_job(bpre, nj);                                                         \
        {                                                                                           \
            const int* src = reinterpret_cast<const int*>(J + jj);                                  \
            int* dst = reinterpret_cast<int*>(&sj);                                                 \
            for (int k = threadIdx.x; k < (int)(sizeof(mel_prox_job) / sizeof(int)); k += blockDim.x) dst[k] = src[k]; \
        }                                                                                           \
        __syncthreads();                                                                            \
        const int it = (blockIdx.x - bpre[jj]) * (PROX_THREADS / (TPI)) + (int)threadIdx.x / (TPI); \
        const int lane = threadIdx.x & 31;                                                          \
        (void)lane;                                                                                 \
        const mel_prox_job& j = sj;                                                                 \
        const mel_dev& d = sj.d;                                                                    \
        (void)j; (void)d;                                                                           \
        __VA_ARGS__;                                                                                \
    }

JOB_KERNEL(aabb_kernel, 32, aabb_item(d, j.aabb, j.shmin, j.shmax, it, lane))
JOB_KERNEL(segblock_kernel, 1, segblock_item(d, it))
JOB_KERNEL(superblock_kernel, 1, superblock_item(d, it))
JOB_KERNEL(neighbour_kernel, 32, neighbour_item(d, j.aabb, j.shmin, j.shmax, j.nbr, j.nbn, j.nbr_cap, it, lane))
JOB_KERNEL(cl_zero_kernel, 1, cl_zero_item(j, it))
JOB_KERNEL(cl_count_kernel, 1, cl_count_item(j, it))
JOB_KERNEL(cl_fill_kernel, 1, cl_fill_item(j, it))
JOB_KERNEL(cl_neighbour_kernel, 32, cl_neighbour_item(j, it, lane))
JOB_KERNEL(task_count_kernel, 1, task_count_item(d, j.nbn, j.tcnt, j.scnt, it))
JOB_KERNEL(zero_tcnt_kernel, 1, if (it <= d.nb) j.tcnt[it] = 0)
JOB_KERNEL(task_fill_kernel, 1, task_fill_item(d, j.nbr, j.nbn, j.nbr_cap, j.btask0, j.bslot0, j.task, j.tns, j.tslot,
                                               j.tkey, j.tcnt, it))
JOB_KERNEL(slot_task_kernel, 32, slot_task_item(d, j.task, j.ntask, j.tmap, it, lane))
JOB_KERNEL(count_kernel, 1, count_item(d, j.task, j.tmap, j.nslot, j.nbr, j.nbr_cap, j.slot_cnt, it))
// slots with candidates: flags in place of the counts (after their scan), then their list
JOB_KERNEL(nz_flag_kernel, 1, if (it < j.nslot) j.slot_cnt[it] = j.slot_cnt[it] > 0 ? 1 : 0)
JOB_KERNEL(nz_list_kernel, 1, if (it < j.nslot && j.slot_cnt[it]) j.nzlist[j.nzoff[it]] = it)
JOB_KERNEL(write_kernel, 1, write_item(d, j.task, j.tmap, j.nzlist, j.nnz, j.nbr, j.nbr_cap, j.slot_off, j.cont_new,
                                       d.cont, j.e_ptr, j.e_list, j.have_old, it))
JOB_KERNEL(zero_contw_kernel, 1, if (it <= d.ncont) d.cont_w[it] = 0.)
JOB_KERNEL(copy_inc_kernel, 1, if (it < d.nb) j.tcnt[it] = j.b_inc0[it])
JOB_KERNEL(inc_fill_kernel, 1, inc_fill_item(j.tkey, j.ntask, j.tcnt, j.inc_task, it))
JOB_KERNEL(inc_sort_kernel, 32, inc_sort_item(d.nb, j.b_inc0, j.inc_task, j.inc_task + j.ntask, it, lane))
JOB_KERNEL(inc_range_kernel, 1, inc_range_item(j.inc_task + j.ntask, j.ntask, j.tslot, j.tns, j.slot_off, j.inc_rng, it))
JOB_KERNEL(body_range_kernel, 1, body_range_item(d.cont, d.ncont, d.nb, j.b_cont0, it))
JOB_KERNEL(zero_ecnt_kernel, 1, if (it <= d.ne) j.e_cnt[it] = 0)
JOB_KERNEL(entry_count_kernel, 1, entry_count_item(d, d.cont, d.ncont, j.e_cnt, it))
JOB_KERNEL(copy_eptr_kernel, 1, if (it <= d.ne) j.e_cur[it] = j.e_ptr[it])
JOB_KERNEL(entry_index_kernel, 32, entry_index_item(d, d.cont, j.b_cont0, j.e_cur, j.e_list, it, lane))
JOB_KERNEL(carry_kernel, 32, carry_item(d, d.cont, j.b_cont0, it, lane))

// one thread per member: clear the neighbour-overflow words before an attempt
__global__ void nbr_clear_kernel(const mel_prox_job* J, int nj)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nj) return;
    J[k].d.err[MEL_E_NBR_OVERFLOW] = 0u;
    J[k].d.err[MEL_E_NBR_NEED] = 0u;
}
// one thread per member: the words the host needs after the neighbour stage (0-4) or the count
// stage (5)
__global__ void readback_kernel(const mel_prox_job* J, int nj, int stage)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nj) return;
    const mel_prox_job& j = J[k];
    int* r = j.readback;
    if (stage == 0) {
        r[0] = (int)j.d.err[MEL_E_NAN];
        r[1] = (int)j.d.err[MEL_E_NBR_OVERFLOW];
        r[2] = (int)j.d.err[MEL_E_NBR_NEED];
        r[3] = j.btask0[j.d.nb];
        r[4] = j.bslot0[j.d.nb];
    } else {
        r[5] = j.slot_off[j.nslot];
        r[6] = j.nzoff[j.nslot];
    }
}

} // namespace mel

// =============================================================================================
// host driver
// =============================================================================================
static int ensure_impl(void** p, size_t* cap_bytes, size_t need, const char* what)
{
    if (need <= *cap_bytes && *p) return 0;
    size_t nc = 2 * need + 4096;            // doubling: few reallocations (each free synchronises the device)
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

// Staging of a run: job tables, block prefixes and scan jobs are written to pinned host memory and
// copied to the same offsets of a device buffer on the run's stream; the space is reused after
// each synchronisation of the stream.  The read-back words of the members live apart.
struct mel_prox_stage {
    char* h = nullptr; char* dv = nullptr; size_t cap = 0, used = 0;
    int* rb_h = nullptr; int* rb_d = nullptr; int rb_cap = 0;    // 8 words per member; rb_d[8 * rb_cap] = 0
    const int* zero = nullptr;     // block prefix of a one-member launch (blocks start at 0)
    std::vector<std::pair<char*, char*>> retired;               // outgrown buffers, freed after a sync
};

static void stage_release_retired(mel_prox_stage& S)
{
    for (auto& b : S.retired) { cudaFreeHost(b.first); cudaFree(b.second); }
    S.retired.clear();
}

void mel_prox_stage_free(mel_prox_stage* S)
{
    if (!S) return;
    stage_release_retired(*S);
    if (S->h) cudaFreeHost(S->h);
    if (S->dv) cudaFree(S->dv);
    if (S->rb_h) cudaFreeHost(S->rb_h);
    if (S->rb_d) cudaFree(S->rb_d);
    delete S;
}

// copies `bytes` from src to the device side of the stage (stream ordered); nullptr on failure
static void* stage_upload(mel_prox_stage& S, const void* src, size_t bytes, cudaStream_t s)
{
    const size_t off = (S.used + 15) & ~(size_t)15;
    if (off + bytes > S.cap) {
        // grow: data already staged may still be read by work on the stream, so the old buffers
        // are kept until the next synchronisation
        size_t nc = 2 * (off + bytes) + (1 << 16);
        char *nh = nullptr, *nd = nullptr;
        if (cudaMallocHost(&nh, nc) != cudaSuccess) return nullptr;
        if (cudaMalloc(&nd, nc) != cudaSuccess) { cudaFreeHost(nh); return nullptr; }
        if (S.h) S.retired.push_back({ S.h, S.dv });
        S.h = nh; S.dv = nd; S.cap = nc;
        S.used = 0;
        return stage_upload(S, src, bytes, s);
    }
    memcpy(S.h + off, src, bytes);
    if (cudaMemcpyAsync(S.dv + off, S.h + off, bytes, cudaMemcpyHostToDevice, s) != cudaSuccess) return nullptr;
    S.used = off + bytes;
    return S.dv + off;
}

namespace {

typedef void (*job_kernel_t)(const mel_prox_job*, const int*, int);

struct run_ctx {
    mel_prox_stage& S;
    cudaStream_t s;
    int launches;
};

// scratch ints of an exclusive scan of n entries (block totals of every level)
size_t scan_scratch_ints(int n)
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

// kernel k over items[j] items of member j of the job table J (TPI threads per item)
int launch_jobs(run_ctx& C, job_kernel_t k, const mel_prox_job* J, const std::vector<int>& items, int tpi)
{
    const int nj = (int)items.size();
    const int per_block = PROX_THREADS / tpi;
    std::vector<int> bpre(nj + 1, 0);
    for (int j = 0; j < nj; j++) bpre[j + 1] = bpre[j] + (items[j] + per_block - 1) / per_block;
    if (bpre[nj] == 0) return MEL_OK;
    const int* dp = nj == 1 ? C.S.zero : (const int*)stage_upload(C.S, bpre.data(), sizeof(int) * (nj + 1), C.s);
    if (!dp) { mel_set_error("proximity staging upload failed"); return MEL_ERR_CUDA; }
    k<<<bpre[nj], PROX_THREADS, 0, C.s>>>(J, dp, nj);
    C.launches++;
    return MEL_OK;
}

// exclusive scans: req[j] scans in[0..n) into out[0..n] using the scratch ws (scan_scratch_ints(n))
struct scan_req { const int* in; int* out; int n; int* ws; };
int scan_many(run_ctx& C, const std::vector<scan_req>& req)
{
    if (req.empty()) return MEL_OK;
    const int nj = (int)req.size();
    std::vector<mel_scan_job> jobs(nj), adds;
    std::vector<int> bpre(nj + 1, 0), apre(1, 0);
    std::vector<scan_req> next;
    for (int j = 0; j < nj; j++) {
        const int nblk = (req[j].n + SCAN_BLOCK) / SCAN_BLOCK;      // covers index n as well
        jobs[j] = { req[j].in, req[j].out, req[j].n, req[j].ws };
        bpre[j + 1] = bpre[j] + nblk;
        if (nblk > 1) {                                              // block totals scanned the same way
            int* soff = req[j].ws + nblk + 1;
            next.push_back({ req[j].ws, soff, nblk, soff + nblk + 2 });
            adds.push_back({ soff, req[j].out, req[j].n + 1, nullptr });
            apre.push_back(apre.back() + nblk);
        }
    }
    const mel_scan_job* dj = (const mel_scan_job*)stage_upload(C.S, jobs.data(), sizeof(mel_scan_job) * nj, C.s);
    const int* db = nj == 1 ? C.S.zero : (const int*)stage_upload(C.S, bpre.data(), sizeof(int) * (nj + 1), C.s);
    if (!dj || !db) { mel_set_error("proximity staging upload failed"); return MEL_ERR_CUDA; }
    mel::scan_block_kernel<<<bpre[nj], SCAN_BLOCK, 0, C.s>>>(dj, db, nj);
    C.launches++;
    if (next.empty()) return MEL_OK;
    if (int rc = scan_many(C, next)) return rc;
    const mel_scan_job* da = (const mel_scan_job*)stage_upload(C.S, adds.data(), sizeof(mel_scan_job) * adds.size(), C.s);
    const int* dap = adds.size() == 1 ? C.S.zero : (const int*)stage_upload(C.S, apre.data(), sizeof(int) * apre.size(), C.s);
    if (!da || !dap) { mel_set_error("proximity staging upload failed"); return MEL_ERR_CUDA; }
    mel::scan_add_kernel<<<apre.back(), SCAN_BLOCK, 0, C.s>>>(da, dap, (int)adds.size());
    C.launches++;
    return MEL_OK;
}

mel_prox_job make_job(const mel_prox_member& m, int* readback)
{
    mel_prox_job j;
    memset(&j, 0, sizeof j);
    const mel_prox_state& P = *m.P;
    j.d = *m.d;
    j.aabb = P.aabb; j.shmin = P.shmin; j.shmax = P.shmax;
    j.nbr = P.nbr; j.nbn = P.nbn; j.nbr_cap = P.nbr_cap;
    j.ntask = P.ntask; j.nslot = P.nslot; j.have_old = m.d->ncont > 0 ? 1 : 0;
    j.task = (int4*)P.task; j.tns = P.tns; j.tslot = P.tslot; j.tkey = P.tkey;
    j.tcnt = P.tcnt; j.btask0 = P.btask0; j.scnt = P.scnt; j.bslot0 = P.bslot0;
    j.slot_cnt = P.slot_cnt; j.slot_off = P.slot_off; j.inc_task = P.inc_task; j.tmap = P.tmap;
    j.nzoff = P.nzoff; j.nzlist = P.nzlist; j.nnz = P.nnz;
    j.inc_rng = P.inc_rng; j.b_inc0 = P.b_inc0; j.b_cont0 = P.b_cont0;
    j.e_cnt = P.e_cnt; j.e_ptr = P.e_ptr; j.e_cur = P.e_cur; j.e_list = P.e_list;
    j.cont_new = P.cont_alt;
    j.readback = readback;
    j.cl_on = P.cl_on; j.cl_T = P.cl_T; j.cl_ncx = P.cl_ncx; j.cl_h = P.cl_h; j.cl_hx = P.cl_hx;
    j.cl_cnt = P.cl_cnt; j.cl_cur = P.cl_cur; j.cl_start = P.cl_start; j.cl_idx = P.cl_idx; j.cl_w = P.cl_w;
    return j;
}

// job table of the members idx (read-back words by member index) on the device
const mel_prox_job* upload_jobs(run_ctx& C, mel_prox_member* m, const std::vector<int>& idx,
                                std::vector<mel_prox_job>& hj)
{
    hj.clear();
    for (int i : idx) hj.push_back(make_job(m[i], C.S.rb_d + 8 * i));
    const mel_prox_job* J = (const mel_prox_job*)stage_upload(C.S, hj.data(), sizeof(mel_prox_job) * hj.size(), C.s);
    if (!J) mel_set_error("proximity staging upload failed");
    return J;
}

template <typename F>
std::vector<int> items_of(const std::vector<mel_prox_job>& hj, F&& f)
{
    std::vector<int> v;
    for (const mel_prox_job& j : hj) v.push_back(f(j));
    return v;
}

// the per-entry index of each member's current list (d.cont, d.ncont) and b_cont0.  The members'
// e_list must hold ncont + 1 entries and their scan scratch scan_scratch_ints(ne); J / hj is the
// job table of the members idx.
int index_stage(run_ctx& C, mel_prox_member* m, const std::vector<int>& idx, const mel_prox_job* J,
                const std::vector<mel_prox_job>& hj)
{
    using namespace mel;
    int rc;
    if ((rc = launch_jobs(C, body_range_kernel, J, items_of(hj, [](const mel_prox_job& j) { return j.d.nb + 1; }), 1))) return rc;
    if ((rc = launch_jobs(C, zero_ecnt_kernel, J, items_of(hj, [](const mel_prox_job& j) { return j.d.ne + 1; }), 1))) return rc;
    if ((rc = launch_jobs(C, entry_count_kernel, J, items_of(hj, [](const mel_prox_job& j) { return j.d.ncont; }), 1))) return rc;
    std::vector<scan_req> sc;
    for (int i : idx) sc.push_back({ m[i].P->e_cnt, m[i].P->e_ptr, m[i].d->ne, m[i].P->scan_ws });
    if ((rc = scan_many(C, sc))) return rc;
    if ((rc = launch_jobs(C, copy_eptr_kernel, J, items_of(hj, [](const mel_prox_job& j) { return j.d.ne + 1; }), 1))) return rc;
    return launch_jobs(C, entry_index_kernel, J, items_of(hj, [](const mel_prox_job& j) { return j.d.nb; }), 32);
}

bool stage_ready(mel_prox_stage*& stage, int n)
{
    if (!stage) stage = new mel_prox_stage();
    mel_prox_stage& S = *stage;
    if (S.rb_cap >= n) return true;
    if (S.rb_h) { cudaFreeHost(S.rb_h); S.rb_h = nullptr; }
    if (S.rb_d) { cudaFree(S.rb_d); S.rb_d = nullptr; }
    S.rb_cap = 0;
    const int cap = std::max(n, 16);
    if (cudaMallocHost(&S.rb_h, sizeof(int) * 8 * (size_t)cap) != cudaSuccess) return false;
    if (cudaMalloc(&S.rb_d, sizeof(int) * (8 * (size_t)cap + 1)) != cudaSuccess) return false;
    if (cudaMemset(S.rb_d, 0, sizeof(int) * (8 * (size_t)cap + 1)) != cudaSuccess) return false;
    S.zero = S.rb_d + 8 * (size_t)cap;
    S.rb_cap = cap;
    return true;
}

// read-back words of members 0..n-1 to the host (one copy, one synchronisation); the stage space is
// free again afterwards
bool read_back(run_ctx& C, int n)
{
    if (cudaMemcpyAsync(C.S.rb_h, C.S.rb_d, sizeof(int) * 8 * (size_t)n, cudaMemcpyDeviceToHost, C.s) != cudaSuccess) return false;
    if (sync_failed(C.s, __LINE__)) return false;
    C.S.used = 0;
    stage_release_retired(C.S);
    return true;
}

}  // namespace

int mel_run_proximity_many(mel_prox_member* m, int n, mel_prox_stage*& stage, int& launches, cudaStream_t s)
{
    using namespace mel;
    if (n <= 0) return MEL_OK;
    if (!stage_ready(stage, n)) { mel_set_error("proximity read-back buffers could not be allocated"); return MEL_ERR_OOM; }
    run_ctx C{ *stage, s, 0 };
    std::vector<mel_prox_job> hj;
    std::vector<int> act;
    int rc;
    for (int i = 0; i < n; i++) {
        m[i].rc = MEL_OK;
        m[i].msg.clear();
        mel_prox_state& P = *m[i].P;
        const int nsc = std::max(m[i].d->nb, m[i].d->ne);
        if (ensure((void**)&P.scan_ws, &P.scan_ws_bytes, sizeof(int) * scan_scratch_ints(std::max(nsc, P.cl_T)))) return MEL_ERR_OOM;
        act.push_back(i);
    }
    // 1. border boxes and segment-block boxes
    const mel_prox_job* J = upload_jobs(C, m, act, hj);
    if (!J) return MEL_ERR_CUDA;
    if ((rc = launch_jobs(C, aabb_kernel, J, items_of(hj, [](const mel_prox_job& j) { return j.d.nbd; }), 32))) return rc;
    if ((rc = launch_jobs(C, segblock_kernel, J, items_of(hj, [](const mel_prox_job& j) { return j.d.nblk; }), 1))) return rc;
    if ((rc = launch_jobs(C, superblock_kernel, J, items_of(hj, [](const mel_prox_job& j) { return j.d.nsblk; }), 1))) return rc;
    // 2. neighbours and the task counts; a member whose neighbour lists overflow grows them and
    //    repeats this stage (up to 4 attempts)
    std::vector<int> pend = act;
    for (int attempt = 0; attempt < 4 && !pend.empty(); attempt++) {
        J = upload_jobs(C, m, pend, hj);
        if (!J) return MEL_ERR_CUDA;
        const int np = (int)pend.size();
        nbr_clear_kernel<<<(np + 127) / 128, 128, 0, s>>>(J, np); C.launches++;
        // members with the cell list: bucket the border boxes (counting sort), then query; the
        // others: all pairs of bodies
        bool any_cl = false, any_ap = false;
        for (const mel_prox_job& jj : hj) { any_cl = any_cl || jj.cl_on; any_ap = any_ap || !jj.cl_on; }
        if (any_cl) {
            if ((rc = launch_jobs(C, cl_zero_kernel, J, items_of(hj, [](const mel_prox_job& j) { return j.cl_on ? j.cl_T + 1 : 0; }), 1))) return rc;
            if ((rc = launch_jobs(C, cl_count_kernel, J, items_of(hj, [](const mel_prox_job& j) { return j.cl_on ? j.d.nbd : 0; }), 1))) return rc;
            std::vector<scan_req> sc;
            for (int i : pend) if (m[i].P->cl_on) sc.push_back({ m[i].P->cl_cnt, m[i].P->cl_start, m[i].P->cl_T, m[i].P->scan_ws });
            if ((rc = scan_many(C, sc))) return rc;
            if ((rc = launch_jobs(C, cl_fill_kernel, J, items_of(hj, [](const mel_prox_job& j) { return j.cl_on ? j.d.nbd : 0; }), 1))) return rc;
            if ((rc = launch_jobs(C, cl_neighbour_kernel, J, items_of(hj, [](const mel_prox_job& j) { return j.cl_on ? j.d.nb : 0; }), 32))) return rc;
        }
        if (any_ap)
            if ((rc = launch_jobs(C, neighbour_kernel, J, items_of(hj, [](const mel_prox_job& j) { return j.cl_on ? 0 : j.d.nb; }), 32))) return rc;
        if ((rc = launch_jobs(C, task_count_kernel, J, items_of(hj, [](const mel_prox_job& j) { return j.d.nb; }), 1))) return rc;
        std::vector<scan_req> sc1, sc2;
        for (int i : pend) {
            sc1.push_back({ m[i].P->tcnt, m[i].P->btask0, m[i].d->nb, m[i].P->scan_ws });
            sc2.push_back({ m[i].P->scnt, m[i].P->bslot0, m[i].d->nb, m[i].P->scan_ws });
        }
        if ((rc = scan_many(C, sc1))) return rc;
        if ((rc = scan_many(C, sc2))) return rc;
        readback_kernel<<<(np + 127) / 128, 128, 0, s>>>(J, np, 0); C.launches++;
        if ((rc = launch_status(__LINE__))) return rc;
        if (!read_back(C, n)) return MEL_ERR_CUDA;
        std::vector<int> retry;
        for (int i : pend) {
            const int* r = C.S.rb_h + 8 * i;
            mel_prox_state& P = *m[i].P;
            if (r[0]) {
                m[i].rc = MEL_ERR_NAN;
                char buf[160];
                if (r[0] & 1) snprintf(buf, sizeof buf, "non-finite node positions at the proximity update");
                else snprintf(buf, sizeof buf, "a border box spans more than %d periods: diverged positions", MEL_MAX_SHIFT_SPAN);
                m[i].msg = buf;
                continue;
            }
            if (r[1]) {
                const int need = r[2] + 16;
                cudaFree(P.nbr); P.nbr = nullptr;
                if (cudaMalloc(&P.nbr, sizeof(int) * 3 * (size_t)need * m[i].d->nb) != cudaSuccess) {
                    mel_set_error("allocation of neighbour lists (%d per body) failed", need);
                    return MEL_ERR_OOM;
                }
                P.nbr_cap = need;
                retry.push_back(i);
                continue;
            }
            P.ntask = r[3];
            P.nslot = r[4];
        }
        pend = retry;
    }
    for (int i : pend) { m[i].rc = MEL_ERR_BOUNDS; m[i].msg = "neighbour lists still over capacity after 4 attempts"; }
    act.clear();
    for (int i = 0; i < n; i++) if (m[i].rc == MEL_OK) act.push_back(i);
    if (act.empty()) { launches += C.launches; return launch_status(__LINE__); }
    // 3. the task list and the candidate count of every slot
    for (int i : act) {
        mel_prox_state& P = *m[i].P;
        const size_t nt = (size_t)P.ntask + 1, ns = (size_t)P.nslot + 1;
        if (ensure((void**)&P.task, &P.task_bytes, sizeof(int4) * nt)) return MEL_ERR_OOM;
        if (ensure((void**)&P.tns, &P.tns_bytes, sizeof(int) * nt)) return MEL_ERR_OOM;
        if (ensure((void**)&P.tslot, &P.tslot_bytes, sizeof(int) * nt)) return MEL_ERR_OOM;
        if (ensure((void**)&P.tkey, &P.tkey_bytes, sizeof(int) * nt)) return MEL_ERR_OOM;
        if (ensure((void**)&P.inc_task, &P.inc_task_bytes, sizeof(int) * 2 * nt)) return MEL_ERR_OOM;
        if (ensure((void**)&P.slot_cnt, &P.slot_bytes, sizeof(int) * ns)) return MEL_ERR_OOM;
        if (ensure((void**)&P.slot_off, &P.slot_off_bytes, sizeof(int) * ns)) return MEL_ERR_OOM;
        if (ensure((void**)&P.tmap, &P.tmap_bytes, sizeof(int) * ns)) return MEL_ERR_OOM;
        if (ensure((void**)&P.nzoff, &P.nzoff_bytes, sizeof(int) * ns)) return MEL_ERR_OOM;
        if (ensure((void**)&P.nzlist, &P.nzlist_bytes, sizeof(int) * ns)) return MEL_ERR_OOM;
        const int nsc = std::max(std::max(m[i].d->nb, m[i].d->ne), P.nslot);
        if (ensure((void**)&P.scan_ws, &P.scan_ws_bytes, sizeof(int) * scan_scratch_ints(std::max(nsc, P.cl_T)))) return MEL_ERR_OOM;
    }
    J = upload_jobs(C, m, act, hj);
    if (!J) return MEL_ERR_CUDA;
    if ((rc = launch_jobs(C, zero_tcnt_kernel, J, items_of(hj, [](const mel_prox_job& j) { return j.d.nb + 1; }), 1))) return rc;
    if ((rc = launch_jobs(C, task_fill_kernel, J, items_of(hj, [](const mel_prox_job& j) { return j.ntask > 0 ? j.d.nb : 0; }), 1))) return rc;
    if ((rc = launch_jobs(C, slot_task_kernel, J, items_of(hj, [](const mel_prox_job& j) { return j.ntask; }), 32))) return rc;
    if ((rc = launch_jobs(C, count_kernel, J, items_of(hj, [](const mel_prox_job& j) { return j.ntask > 0 ? j.nslot : 0; }), 1))) return rc;
    {
        std::vector<scan_req> sc, sz;
        for (int i : act) {
            sc.push_back({ m[i].P->slot_cnt, m[i].P->slot_off, m[i].P->nslot, m[i].P->scan_ws });
            sz.push_back({ m[i].P->slot_cnt, m[i].P->nzoff, m[i].P->nslot, m[i].P->scan_ws });
        }
        if ((rc = scan_many(C, sc))) return rc;
        // the write pass visits only the slots with candidates (a few in a thousand)
        if ((rc = launch_jobs(C, nz_flag_kernel, J, items_of(hj, [](const mel_prox_job& j) { return j.ntask > 0 ? j.nslot : 0; }), 1))) return rc;
        if ((rc = scan_many(C, sz))) return rc;
        if ((rc = launch_jobs(C, nz_list_kernel, J, items_of(hj, [](const mel_prox_job& j) { return j.ntask > 0 ? j.nslot : 0; }), 1))) return rc;
    }
    readback_kernel<<<((int)act.size() + 127) / 128, 128, 0, s>>>(J, (int)act.size(), 1); C.launches++;
    if ((rc = launch_status(__LINE__))) return rc;
    if (!read_back(C, n)) return MEL_ERR_CUDA;
    // 4. the new list, written into the spare buffer with history inherited from the current one
    for (int i : act) {
        mel_prox_state& P = *m[i].P;
        const size_t total = (size_t)C.S.rb_h[8 * i + 5];
        P.nnz = C.S.rb_h[8 * i + 6];
        if (ensure((void**)&P.cont_alt, &P.cont_alt_bytes, sizeof(mel_contact) * (total + 1))) return MEL_ERR_OOM;
        if (ensure((void**)&P.cont_w, &P.cont_w_bytes, sizeof(double) * (total + 1))) return MEL_ERR_OOM;
        if (ensure((void**)&P.cont_rt, &P.cont_rt_bytes, 6 * sizeof(double) * (total + 1))) return MEL_ERR_OOM;
        if (ensure((void**)&P.inc_rng, &P.inc_rng_bytes, sizeof(int2) * ((size_t)P.ntask + 1))) return MEL_ERR_OOM;
    }
    J = upload_jobs(C, m, act, hj);
    if (!J) return MEL_ERR_CUDA;
    if ((rc = launch_jobs(C, write_kernel, J, items_of(hj, [](const mel_prox_job& j) { return j.ntask > 0 ? j.nnz : 0; }), 1))) return rc;
    for (int i : act) {
        mel_dev& d = *m[i].d;
        mel_prox_state& P = *m[i].P;
        mel_contact* old = d.cont;
        const size_t old_bytes = P.cont_bytes;
        d.cont = P.cont_alt; P.cont_bytes = P.cont_alt_bytes;
        P.cont_alt = old; P.cont_alt_bytes = old_bytes;
        d.ncont = C.S.rb_h[8 * i + 5];
        d.cont_w = P.cont_w;
        d.cont_rt = P.cont_rt;
        d.inc_rng = P.inc_rng;
        d.b_inc0 = P.b_inc0;
        d.b_cont0 = P.b_cont0;
        // the old index is read by the write pass just launched; freeing it waits for that pass
        if (ensure((void**)&P.e_list, &P.e_list_bytes, sizeof(int) * ((size_t)d.ncont + 1))) return MEL_ERR_OOM;
    }
    J = upload_jobs(C, m, act, hj);
    if (!J) return MEL_ERR_CUDA;
    if ((rc = launch_jobs(C, zero_contw_kernel, J, items_of(hj, [](const mel_prox_job& j) { return j.d.ncont + 1; }), 1))) return rc;
    // 5. incoming ranges in send order
    {
        std::vector<scan_req> sc;
        for (int i : act) sc.push_back({ m[i].P->tcnt, m[i].P->b_inc0, m[i].d->nb, m[i].P->scan_ws });
        if ((rc = scan_many(C, sc))) return rc;
    }
    if ((rc = launch_jobs(C, copy_inc_kernel, J, items_of(hj, [](const mel_prox_job& j) { return j.ntask > 0 ? j.d.nb : 0; }), 1))) return rc;
    if ((rc = launch_jobs(C, inc_fill_kernel, J, items_of(hj, [](const mel_prox_job& j) { return j.ntask; }), 1))) return rc;
    if ((rc = launch_jobs(C, inc_sort_kernel, J, items_of(hj, [](const mel_prox_job& j) { return j.ntask > 0 ? j.d.nb : 0; }), 32))) return rc;
    if ((rc = launch_jobs(C, inc_range_kernel, J, items_of(hj, [](const mel_prox_job& j) { return j.ntask; }), 1))) return rc;
    // 6. per-entry index of the new list; vgapn/vgapt carry of new elements
    if ((rc = index_stage(C, m, act, J, hj))) return rc;
    if ((rc = launch_jobs(C, carry_kernel, J, items_of(hj, [](const mel_prox_job& j) { return j.d.nb; }), 32))) return rc;
    launches += C.launches;
    return launch_status(__LINE__);
}

int mel_run_proximity(mel_dev& d, mel_prox_state& P, const mel_prox_host& H, cudaStream_t s)
{
    (void)H;
    mel_prox_member m;
    m.d = &d;
    m.P = &P;
    int launches = 0;
    const int rc = mel_run_proximity_many(&m, 1, P.stage, launches, s);
    P.launches += launches;
    if (rc) return rc;
    if (m.rc) { mel_set_error("%s", m.msg.c_str()); return m.rc; }
    return MEL_OK;
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
    d.b_cont0 = P.b_cont0;
    if (ensure((void**)&P.e_list, &P.e_list_bytes, sizeof(int) * ((size_t)d.ncont + 1))) return MEL_ERR_OOM;
    if (ensure((void**)&P.scan_ws, &P.scan_ws_bytes, sizeof(int) * scan_scratch_ints(std::max(std::max(d.nb, d.ne), P.cl_T)))) return MEL_ERR_OOM;
    if (!stage_ready(P.stage, 1)) { mel_set_error("proximity read-back buffers could not be allocated"); return MEL_ERR_OOM; }
    mel_prox_member m;
    m.d = &d;
    m.P = &P;
    run_ctx C{ *P.stage, s, 0 };
    std::vector<mel_prox_job> hj;
    const std::vector<int> idx{ 0 };
    const mel_prox_job* J = upload_jobs(C, &m, idx, hj);
    if (!J) return MEL_ERR_CUDA;
    int rc = index_stage(C, &m, idx, J, hj);
    P.launches += C.launches;
    if (rc) return rc;
    if (sync_failed(s, __LINE__)) return MEL_ERR_CUDA;
    C.S.used = 0;
    stage_release_retired(C.S);
    return launch_status(__LINE__);
}
