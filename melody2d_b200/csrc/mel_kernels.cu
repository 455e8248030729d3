// Step kernels of the B200 solver.
//
//   contact_kernel  one thread per contact element: Body::Update_contacts (Code/Body.h:1341-1634)
//                   for that element, the slave border length of Body::Update_borders
//                   (Code/Body.h:614-661) and the contact law of Body::Update_contact_forces
//                   (Code/Body.h:1642-1849); extra threads refresh every border entry's length.
//   body_kernel     one CTA per body: Update_bc_forces, Update_body_forces, the contact force
//                   scatter of Update_contact_forces + Send_contact_forces (Code/Body.h:1855-1967),
//                   Update_internal_forces (Code/Body.h:937-1049), Sum_up_forces, Apply_Newton,
//                   Update_bc(t+dt), Apply_Euler, Update_kinematics, Update_current_positions.
//
// Every floating-point accumulation keeps the reference's order (Gauss points ascending for the
// internal forces, contact list order then send order for contact forces), so with identical inputs
// the FP64 path reproduces the reference's values exactly; this file is compiled with
// -fmad=false.
#include <cstdio>
#include <mutex>
#include "mel_internal.h"
#include "mel_geometry.cuh"
#include "mel_sincos.h"

namespace mel {

__device__ __forceinline__ void set_err(const mel_dev& d, int w, unsigned v = 1u) { atomicOr(&d.err[w], v); }

// pow(x, p) of the mass-scaling increments (Code/Node.h:280, Code/Body.h:2576).  For the exponents 1,
// 2 and 1/2 the correctly rounded value is x, x*x and sqrt(x), which is what glibc's pow returns;
// other exponents go through CUDA's pow, whose last bit can differ from glibc's.
__device__ __forceinline__ double ms_pow(double x, double p)
{
    if (p == 1.) return x;
    if (p == 2.) return x * x;
    if (p == 0.5) return sqrt(x);
    return pow(x, p);
}

// Body::Update_borders length of entry j of global border g of deformable body b
__device__ __forceinline__ double border_length(const mel_dev& d, int b, int g, int j)
{
    int e = d.bd_e0[g] + j;
    int nbn = d.bd_e0[g + 1] - d.bd_e0[g];
    int n0 = d.b_node0[b];
    const int* sn = d.e_sn + 4 * e;
    const int* ss = d.e_ss + 4 * e;
    double2 p0 = d.x[n0 + sn[0]], p1 = d.x[n0 + sn[1]], p2 = d.x[n0 + sn[2]];
    double x0 = p0.x + d.period * ss[0], y0 = p0.y;
    double x1 = p1.x + d.period * ss[1], y1 = p1.y;
    double x2 = p2.x + d.period * ss[2], y2 = p2.y;
    bool simple = d.bd_per[g] == MEL_PER_SIMPLE;
    if (j == 0 && simple) return sqrt((x2 - x1) * (x2 - x1) + (y2 - y1) * (y2 - y1)) * 0.5;
    if (j == nbn - 1 && simple) return sqrt((x1 - x0) * (x1 - x0) + (y1 - y0) * (y1 - y0)) * 0.5;
    return (sqrt((x2 - x1) * (x2 - x1) + (y2 - y1) * (y2 - y1)) + sqrt((x1 - x0) * (x1 - x0) + (y1 - y0) * (y1 - y0))) * 0.5;
}

__device__ __forceinline__ double entry_length(const mel_dev& d, int b, int g, int j)
{
    if (d.b_type[b] == MEL_BODY_DEFORMABLE) return border_length(d, b, g, j);
    return d.e_len0[d.bd_e0[g] + j];
}

// ------------------------------------------------------------------------------------------
// contact kernel
// ------------------------------------------------------------------------------------------
__device__ __forceinline__ void seg_points(const mel_dev& d, int bodyM, int e, int shiftM, int* nd, int* sh,
                                           double* X, double* Y)
{
    int mb = d.b_node0[bodyM];
    for (int k = 0; k < 4; k++) {
        nd[k] = d.e_sn[4 * e + k];
        sh[k] = d.e_ss[4 * e + k];
        double2 p = d.x[mb + nd[k]];
        X[k] = p.x + d.period * (shiftM + sh[k]);
        Y[k] = p.y;
    }
}

// Moment-arm terms of one contact for rigid bodies (Body::Update_contact_forces, rigid branches,
// Code/Body.h:1866-1877 and the master side read by Sum_up_forces): the slave side adds
// (fx, fy, -fx*dy + fy*dx) to a rigid slave, the master side (-fx, -fy, fx*dy - fy*dx) to a rigid
// master, with arms from the body centre to the slave node.  Contacts whose material pair has no
// law contribute +0, which leaves the body's running sums unchanged.  Written here, where every
// contact is one thread, so the rigid body only adds them up in the reference's order.
__device__ __forceinline__ void rigid_terms(const mel_dev& d, int tid, const mel_contact& c, double2 xs)
{
    double* t = d.cont_rt + 6 * (size_t)tid;
    const bool law = d.table[d.b_mat[c.bodyS] * d.nmat + d.b_mat[c.bodyM]] > -1;
    if (d.b_type[c.bodyS] == MEL_BODY_RIGID) {
        const double* rg = d.rg + MEL_RIGID_NF * c.bodyS;
        double dx = xs.x - rg[MEL_RG_XC], dy = xs.y - rg[MEL_RG_YC];
        t[0] = law ? c.fx : 0.;
        t[1] = law ? c.fy : 0.;
        t[2] = law ? -c.fx * dy + c.fy * dx : 0.;
    }
    if (d.b_type[c.bodyM] == MEL_BODY_RIGID) {
        const double* rg = d.rg + MEL_RIGID_NF * c.bodyM;
        double dx = xs.x - rg[MEL_RG_XC] - c.shiftM * d.period;
        double dy = xs.y - rg[MEL_RG_YC];
        t[3] = law ? -c.fx : 0.;
        t[4] = law ? -c.fy : 0.;
        t[5] = law ? c.fx * dy - c.fy * dx : 0.;
    }
}

// one thread of the contact pass: contact element `tid`, or border entry tid - ncont.  With
// czm_init the pass is Initialize_CZM's instead (Code/Proximity.h:481-541): the contact geometry is
// updated as in Update_contacts, then contacts whose law has bonds start bonded when their gap is
// below the law's initial-gap parameter; no law is evaluated and no force is written.
__device__ void contact_thread(const mel_dev& d, int tid, double law_dt_scale, int czm_init = 0)
{
    if (tid >= d.ncont) {
        if (czm_init) return;
        // refresh stored border lengths (read by Update_proximity for new contacts)
        int e = tid - d.ncont;
        if (e >= d.ne) return;
        // find the border of entry e: binary search on bd_e0
        int lo = 0, hi = d.nbd;
        while (hi - lo > 1) { int mid = (lo + hi) >> 1; if (d.bd_e0[mid] <= e) lo = mid; else hi = mid; }
        int b = d.bd_body[lo];
        if (d.b_status[b] == MEL_STATUS_INACTIVE) return;
        if (d.b_type[b] == MEL_BODY_DEFORMABLE) d.e_len[e] = border_length(d, b, lo, e - d.bd_e0[lo]);
        return;
    }
    mel_contact c = d.cont[tid];
    int b = c.bodyS;
    if (b < 0 || b >= d.nb || c.bodyM < 0 || c.bodyM >= d.nb) { set_err(d, MEL_E_BOUNDS); return; }
    if (d.b_status[b] == MEL_STATUS_INACTIVE) {
        if (!czm_init) rigid_terms(d, tid, c, d.x[d.b_node0[b] + c.nodeS]);
        return;
    }
    // ---- Update_contacts (Code/Body.h:1352-1632) -----------------------------------------
    int bodyM = c.bodyM, borderM = c.borderM, shiftM = c.shiftM, segmentM = c.segmentM;
    int gM = d.b_bd0[bodyM] + borderM;
    int per = d.bd_per[gM];
    Proj p;
    p.gap = c.gapn; p.xsi = c.xsi; p.xn = c.xnorm; p.yn = c.ynorm; p.xt = c.xtan; p.yt = c.ytan;
    p.N[0] = c.shapeM[0]; p.N[1] = c.shapeM[1]; p.N[2] = c.shapeM[2]; p.N[3] = c.shapeM[3];
    p.flag = 0;
    double gapt = c.gapt;
    int nd[4], sh[4];
    double X[4], Y[4];
    int e = d.bd_e0[gM] + segmentM;
    seg_points(d, bodyM, e, shiftM, nd, sh, X, Y);
    double xsi_previous = p.xsi;
    int s0 = d.b_node0[b] + c.nodeS;
    double2 xs = d.x[s0];
    bool self1 = (b == bodyM && (nd[0] == c.nodeS || nd[3] == c.nodeS));
    if (self1) closest_self(xs.x, xs.y, X[1], Y[1], X[2], Y[2], p);
    else closest_linear(xs.x, xs.y, X[0], Y[0], X[1], Y[1], X[2], Y[2], X[3], Y[3], p);
    bool set1 = !self1 && (p.flag >= -2 && p.flag <= 2);
    if (p.flag == -2 || p.flag == -3 || p.flag == 2 || p.flag == 3) {
        bool back = (p.flag == -2 || p.flag == -3);
        double L = sqrt((X[2] - X[1]) * (X[2] - X[1]) + (Y[2] - Y[1]) * (Y[2] - Y[1]));
        if (back) gapt = gapt + 0.5 * (-1. - xsi_previous) * L;
        else gapt = gapt + 0.5 * (-1. + xsi_previous) * L;
        int gb = gM;
        int nseg = d.bd_e0[gb + 1] - d.bd_e0[gb] - 2;       // index of the last segment
        if (back) {
            if (per == MEL_PER_SIMPLE) {
                if (segmentM == 0) { borderM = d.bd_bef[gb]; gb = d.b_bd0[bodyM] + borderM; segmentM = d.bd_e0[gb + 1] - d.bd_e0[gb] - 2; }
                else segmentM--;
            } else if (per == MEL_PER_PERIODIC) {
                if (segmentM == 0) {
                    if (borderM == 0) shiftM--; else if (borderM == 1) shiftM++;
                    segmentM = nseg;
                } else segmentM--;
            } else {
                if (segmentM == 0) segmentM = nseg; else segmentM--;
            }
        } else {
            if (per == MEL_PER_SIMPLE) {
                if (segmentM == nseg) { borderM = d.bd_aft[gb]; gb = d.b_bd0[bodyM] + borderM; segmentM = 0; }
                else segmentM++;
            } else if (per == MEL_PER_PERIODIC) {
                if (segmentM == nseg) { if (borderM == 0) shiftM++; else if (borderM == 1) shiftM--; segmentM = 0; }
                else segmentM++;
            } else {
                if (segmentM == nseg) segmentM = 0; else segmentM++;
            }
        }
        gM = d.b_bd0[bodyM] + borderM;
        e = d.bd_e0[gM] + segmentM;
        seg_points(d, bodyM, e, shiftM, nd, sh, X, Y);
        p.xsi = back ? 1. : -1.;
        bool self2 = (b == bodyM && (nd[0] == c.nodeS || nd[3] == c.nodeS));
        if (self2) closest_self(xs.x, xs.y, X[1], Y[1], X[2], Y[2], p);
        else closest_linear(xs.x, xs.y, X[0], Y[0], X[1], Y[1], X[2], Y[2], X[3], Y[3], p);
        bool set2 = !self2 && (p.flag >= -2 && p.flag <= 2);
        if (!set1 && !set2) set_err(d, MEL_E_STALE);   // the reference would reuse another contact's weights
        double L2 = sqrt((X[2] - X[1]) * (X[2] - X[1]) + (Y[2] - Y[1]) * (Y[2] - Y[1]));
        if (back) gapt = gapt + 0.5 * (-1. + p.xsi) * L2;
        else gapt = gapt + 0.5 * (1. + p.xsi) * L2;
        c.bodyM = bodyM; c.borderM = borderM; c.shiftM = shiftM; c.segmentM = segmentM;
    } else {
        gapt = gapt + 0.5 * (p.xsi - xsi_previous) * sqrt((X[2] - X[1]) * (X[2] - X[1]) + (Y[2] - Y[1]) * (Y[2] - Y[1]));
    }
    int mb = d.b_node0[bodyM];
    double2 vs = d.v[s0];
    double2 v0 = d.v[mb + nd[0]], v1 = d.v[mb + nd[1]], v2 = d.v[mb + nd[2]], v3 = d.v[mb + nd[3]];
    double vgapx = vs.x - (p.N[0] * v0.x + p.N[1] * v1.x + p.N[2] * v2.x + p.N[3] * v3.x);
    double vgapy = vs.y - (p.N[0] * v0.y + p.N[1] * v1.y + p.N[2] * v2.y + p.N[3] * v3.y);
    double vgapn = vgapx * p.xn + vgapy * p.yn;
    double vgapt = vgapx * p.xt + vgapy * p.yt;
    for (int k = 0; k < 4; k++) { c.nodeM[k] = nd[k]; c.shiftMk[k] = sh[k]; c.shapeM[k] = p.N[k]; }
    c.xsi = p.xsi; c.xnorm = p.xn; c.ynorm = p.yn; c.xtan = p.xt; c.ytan = p.yt;
    c.vgapn = vgapn; c.vgapt = vgapt;
    if (czm_init) {
        c.gapn = p.gap; c.gapt = gapt;
        const int lb = d.table[d.b_mat[b] * d.nmat + d.b_mat[bodyM]];
        if (lb > -1) {
            const int t = d.law_type[lb];
            const double* P = d.law_p + MEL_LAW_NPARAM * lb;
            if (t == MEL_LAW_CZM_LINEAR) { c.nb_internal = 1; c.internal[0] = (c.gapn < P[5]) ? 0. : 1.; }
            else if (t == MEL_LAW_CZM_FATIGUE || t == MEL_LAW_BONDED_MOHR_COULOMB) {
                const double gi = (t == MEL_LAW_CZM_FATIGUE) ? P[8] : P[10];
                c.nb_internal = 3; c.internal[0] = (c.gapn < gi) ? 0. : 1.; c.internal[1] = 0.; c.internal[2] = 0.;
            }
        }
        d.cont[tid] = c;
        return;
    }
    // ---- Update_contact_forces (Code/Body.h:1657-1849) ----------------------------------
    int gS = d.b_bd0[b] + c.borderS;
    double length = entry_length(d, b, gS, c.border_nodeS);
    double initial_length = d.e_len0[d.bd_e0[gS] + c.border_nodeS];
    double gapn = p.gap;
    int li = d.table[d.b_mat[b] * d.nmat + d.b_mat[bodyM]];
    if (li > -1) {
        double W = 0., Pn = 0., Pt = 0.;
        int nbi = c.nb_internal;
        apply_law(d.law_type[li], d.law_p + MEL_LAW_NPARAM * li, c.effective_mass, initial_length, gapn, vgapn, gapt,
                  vgapt, Pn, Pt, W, nbi, c.internal);
        c.nb_internal = nbi;
        double Px = p.xn * Pn + p.xt * Pt, Py = p.yn * Pn + p.yt * Pt;
        double Fsx, Fsy;
        double dtl = d.dt[0] * law_dt_scale;
        if (d.law_len[li] == MEL_LENGTH_FIXED) { Fsx = Px * initial_length; Fsy = Py * initial_length; W *= initial_length * dtl; }
        else { Fsx = Px * length; Fsy = Py * length; W *= length * dtl; }
        c.length = length; c.fx = Fsx; c.fy = Fsy;
        c.gapn = gapn; c.gapt = gapt;
        d.cont[tid] = c;
        d.cont_w[tid] = W;     // work increment, summed per body in the reference's order by body_kernel
        rigid_terms(d, tid, c, xs);
        return;
    }
    // no law for this material pair: Update_contacts ran, forces untouched (Code/Body.h:1700-1701)
    c.gapn = gapn; c.gapt = gapt;
    d.cont[tid] = c;
    d.cont_w[tid] = 0.;
    rigid_terms(d, tid, c, xs);
}

// ------------------------------------------------------------------------------------------
// boundary-condition histories (Code/Border.h:120-215, Code/Body.h:335-395)
// ------------------------------------------------------------------------------------------
__device__ void border_bc_value(const mel_dev& d, int g, int dir, double T, double& val, double& vel)
{
    int t = d.bd_bc[2 * g + dir];
    int h0 = d.bd_h0[2 * g + dir], h1 = d.bd_h0[2 * g + dir + 1];
    const double* ti = d.ht + h0;
    const double* va = d.hv + h0;
    int nh = h1 - h0;
    val = 0.; vel = 0.;
    if (t == MEL_BC_SOFT) {
        int n = 0, ex = 0;
        double v = 0.;
        while (ex == 0 && n + 1 < nh) {
            double t0 = ti[n], p0 = va[n], t1 = ti[n + 1], p1 = va[n + 1];
            if (T >= t1) v = v + (t1 - t0) * (p1 + p0) * 0.5;
            else { v = v + (T - t0) * (p0 + (p1 - p0) / (t1 - t0) * ((T - t0) * 0.5)); vel = p0 + (p1 - p0) / (t1 - t0) * (T - t0); ex = 1; }
            n++;
        }
        val = v;
    } else if (t == MEL_BC_ORIENTED || t == MEL_BC_FOLLOWING) {
        for (int n = 0; n + 1 < nh; n++) {
            double t0 = ti[n], p0 = va[n], t1 = ti[n + 1], p1 = va[n + 1];
            if ((t0 <= T) & (T <= t1)) { val = p0 + (p1 - p0) / (t1 - t0) * (T - t0); break; }
        }
    }
}

// drivendof of Body::Update_bc for one body at time T (drv[8] updated in place)
__device__ void body_drivendof(const mel_dev& d, int b, double T, double* drv)
{
    for (int n = d.b_bd0[b]; n < d.b_bd0[b + 1]; n++) {
        for (int dir = 0; dir < 2; dir++) {
            if (d.bd_bc[2 * n + dir] != MEL_BC_DRIVEN) continue;
            int h0 = d.bd_h0[2 * n + dir], nh = d.bd_h0[2 * n + dir + 1] - h0;
            const double* ti = d.ht + h0;
            const double* va = d.hv + h0;
            int base = 4 * dir;
            drv[base] = 1.;
            drv[base + 1] = 0.;
            int ex = 0, k = 0;
            while (ex == 0 && k + 1 < nh) {
                double t0 = ti[k], p0 = va[k], t1 = ti[k + 1], p1 = va[k + 1];
                if (T >= t1) drv[base + 1] += (t1 - t0) * (p1 + p0) * 0.5;
                else {
                    drv[base + 1] += (T - t0) * (p0 + (p1 - p0) / (t1 - t0) * ((T - t0) * 0.5));
                    drv[base + 2] = (T - t0) * (p1 - p0) / (t1 - t0);
                    drv[base + 3] = (p1 - p0) / (t1 - t0);
                    ex = 1;
                }
                k++;
            }
        }
    }
}

// ------------------------------------------------------------------------------------------
// body kernel: deformable path
// ------------------------------------------------------------------------------------------
// scatter v * N_j onto the supports of body-local node `node` (one warp; lanes over supports)
__device__ __forceinline__ void warp_scatter(const mel_dev& d, int n0, int node, double fx, double fy, double2* acc, int lane,
                                             int nlanes = 32)
{
    int gn = n0 + node;
    int a = d.sup_ptr[gn], bnd = d.sup_ptr[gn + 1];
    for (int j = a + lane; j < bnd; j += nlanes) {
        double N = d.sup_N[j];
        int t = d.sup_idx[j];
        double2 f = acc[t];
        f.x = f.x + fx * N;
        f.y = f.y + fy * N;
        acc[t] = f;
    }
}

// ---- bulk copies into shared memory and their mbarriers (PTX: mbarrier.*, cp.async.bulk) --
__device__ __forceinline__ unsigned smem_u32(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" :: "r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_init_fence() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, unsigned bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" :: "r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, unsigned parity)
{
    unsigned ok;
    asm volatile("{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n}"
                 : "=r"(ok) : "r"(smem_u32(bar)), "r"(parity) : "memory");
    return ok != 0;
}
__device__ __forceinline__ void bulk_load(void* dst, const void* src, unsigned bytes, uint64_t* bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                 :: "r"(smem_u32(dst)), "l"(src), "r"(bytes), "r"(smem_u32(bar)) : "memory");
}
// generic-proxy accesses to a buffer are ordered before the bulk copy that refills it
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
#define MEL_BODY_CTHREADS 224     // the FP64 kernel's Gauss-point warps (0-6); warp 7 scatters contacts
// barrier of the FP64 kernel's Gauss-point warps only (warp 7 runs the contact scatter meanwhile)
__device__ __forceinline__ void compute_sync() { asm volatile("bar.sync 1, %0;" :: "n"(MEL_BODY_CTHREADS) : "memory"); }
__device__ __forceinline__ void mbar_arrive(uint64_t* bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" :: "r"(smem_u32(bar)) : "memory");
}
// barrier of the pull warps alone (named barrier 3), returning whether any of them passed `v`
template <int NT>
__device__ __forceinline__ bool pull_group_any(bool v)
{
    unsigned r;
    asm volatile("{\n\t.reg .pred p, q;\n\tsetp.ne.u32 p, %1, 0;\n\tbar.red.or.pred q, 3, %2, p;\n\tselp.u32 %0, 1, 0, q;\n}"
                 : "=r"(r) : "r"((unsigned)v), "n"(NT) : "memory");
    return r != 0;
}
// barrier of warps 1-7 in the body tail (warp 0 sums the works meanwhile)
__device__ __forceinline__ void tail_sync() { asm volatile("bar.sync 2, %0;" :: "n"(MEL_BODY_THREADS - 32) : "memory"); }
__device__ __forceinline__ unsigned long long global_ns()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
// wait for phase `parity` of `bar` to complete; gives up after `limit_ns` (the pipeline's waits use
// mel_dev::wait_ns, MEL_WAIT_NS unless a test shortens it; the final wait for copies in flight
// always allows MEL_WAIT_NS)
__device__ __forceinline__ bool mbar_test_wait(uint64_t* bar, unsigned parity)
{
    unsigned ok;
    asm volatile("{\n\t.reg .pred p;\n\tmbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n}"
                 : "=r"(ok) : "r"(smem_u32(bar)), "r"(parity) : "memory");
    return ok != 0;
}
__device__ bool mbar_wait_bounded(uint64_t* bar, unsigned parity, unsigned long long limit_ns = MEL_WAIT_NS)
{
    if (limit_ns == 0) return mbar_test_wait(bar, parity);     // no waiting at all (tests)
    if (mbar_try_wait(bar, parity)) return true;
    const unsigned long long t0 = global_ns();
    while (true) {
        for (int i = 0; i < 64; i++)
            if (mbar_try_wait(bar, parity)) return true;
        if (global_ns() - t0 > limit_ns) return false;
    }
}

// running sums of `n` terms t[k*stride] (k = 0..n-1) added in order to acc; loads batched so
// that eight are in flight per round trip
__device__ __forceinline__ double ordered_sum(double acc, const double* t, int n, int stride)
{
    int k = 0;
    for (; k + 8 <= n; k += 8) {
        double v[8];
#pragma unroll
        for (int j = 0; j < 8; j++) v[j] = t[(size_t)(k + j) * stride];
#pragma unroll
        for (int j = 0; j < 8; j++) acc += v[j];
    }
    for (; k < n; k++) acc += t[(size_t)k * stride];
    return acc;
}

// Gauss-point pass of one chunk held in shared memory (Body::Update_internal_forces,
// Code/Body.h:960-1050): thread `t` < ngp forms the strain of its point from the staged dN and
// the body's displacements (supports in the point's own order), applies the material and
// overwrites its dN pairs with the contributions c0 * B^T.sigma.  The slot's group of m slots
// stores row k of all its slots at base + m k (rows padded to the group's largest point with zero
// derivatives on node 0), lane j's entry at j ^ (k & 7) in rows whose width is a multiple of 8:
// every position is computed, so a support's loads depend on nothing but its own index.
struct mel_rows { int base, m, sw, lane, ns; };
__device__ __forceinline__ mel_rows point_rows(int t, int ngp, const unsigned* s_gpm, const uint16_t* s_roff)
{
    const unsigned gm = s_gpm[t];
    mel_rows R;
    R.base = (int)(s_roff[gm & 0x3ffu] & 0xfffu);
    R.m = min(32, ngp - (t & ~31));
    R.sw = (R.m & 7) == 0 ? 7 : 0;
    R.lane = (int)((gm >> 10) & 0x1fu);
    R.ns = (int)(gm >> 15);
    return R;
}
#define E(k) (R.base + R.m * (k) + (R.lane ^ ((k) & R.sw)))

__device__ __forceinline__ void chunk_points(int t, int ngp, int mtype, double Mu, double Lam, const double2* s_up,
                                             double2* s_p, const uint16_t* s_idx, const double* s_c0,
                                             const unsigned* s_gpm, const uint16_t* s_roff)
{
    const mel_rows R = point_rows(t, ngp, s_gpm, s_roff);
    const int ns = R.ns;
    const double c0 = s_c0[t];
    if (mtype == MEL_MAT_ELASTIC_LINEAR) {
        // strain sums in support order; loads issued eight supports ahead of the adds
        double E11 = 0., E12 = 0., E22 = 0.;
        int k = 0;
        for (; k + 8 <= ns; k += 8) {
            double2 dN[8], u[8];
#pragma unroll
            for (int j = 0; j < 8; j++) { const int e = E(k + j); dN[j] = s_p[e]; u[j] = s_up[s_idx[e]]; }
#pragma unroll
            for (int j = 0; j < 8; j++) {
                E11 = E11 + dN[j].x * u[j].x;
                E12 = E12 + (dN[j].x * u[j].y + dN[j].y * u[j].x);
                E22 = E22 + dN[j].y * u[j].y;
            }
        }
        if (k < ns) {                   // the last rows: loads of up to eight issued together
            double2 dN[8], u[8];
#pragma unroll
            for (int j = 0; j < 8; j++)
                if (k + j < ns) { const int e = E(k + j); dN[j] = s_p[e]; u[j] = s_up[s_idx[e]]; }
#pragma unroll
            for (int j = 0; j < 8; j++)
                if (k + j < ns) {
                    E11 = E11 + dN[j].x * u[j].x;
                    E12 = E12 + (dN[j].x * u[j].y + dN[j].y * u[j].x);
                    E22 = E22 + dN[j].y * u[j].y;
                }
        }
        E12 = 0.5 * E12;
        double J = 1. + E11 + E22;               // Apply_Elastic_Linear (Code/Model.h:19-29)
        double S33 = Lam * (J - 1.);
        double Mu2 = 2 * Mu;
        double S11 = S33 + Mu2 * E11, S22 = S33 + Mu2 * E22, S12 = Mu2 * E12;
#pragma unroll 8
        for (int k2 = 0; k2 < ns; k2++) {
            const int e = E(k2);
            const double2 dN = s_p[e];
            double2 q;
            q.x = c0 * (dN.x * S11 + dN.y * S12);
            q.y = c0 * (dN.y * S22 + dN.x * S12);
            s_p[e] = q;
        }
    } else {
        double F11 = 1., F12 = 0., F21 = 0., F22 = 1.;
        for (int k = 0; k < ns; k++) {
            double2 dN = s_p[E(k)];
            double2 u = s_up[s_idx[E(k)]];
            F11 += dN.x * u.x; F12 += dN.y * u.x; F21 += dN.x * u.y; F22 += dN.y * u.y;
        }
        double Kappa = Lam;                       // Apply_NeoHookean (Code/Model.h:52-73)
        double F11F12 = F11 * F11 + F12 * F12, F21F22 = F21 * F21 + F22 * F22;
        double J = F11 * F22 - F12 * F21;
        double invJ = 1. / J;
        double K = Kappa * (J - 1.);
        double MuJ53 = Mu * pow(J, -1.666666666667);
        double trB = 0.333333333333 * (F11F12 + F21F22 + 1.);
        double s11 = K + MuJ53 * (F11F12 - trB), s22 = K + MuJ53 * (F21F22 - trB);
        double s12 = MuJ53 * (F11 * F21 + F12 * F22);
        double S11 = (F12 * (F12 * s22 - F22 * s12) - F22 * (F12 * s12 - F22 * s11)) * invJ;
        double S22 = (F11 * (F11 * s22 - F21 * s12) - F21 * (F11 * s12 - F21 * s11)) * invJ;
        double S12 = (F21 * (F12 * s12 - F22 * s11) - F11 * (F12 * s22 - F22 * s12)) * invJ;
        for (int k = 0; k < ns; k++) {
            double2 dN = s_p[E(k)];
            double2 q;
            q.x = c0 * (dN.x * (F11 * S11 + F12 * S12) + dN.y * (F12 * S22 + F11 * S12));
            q.y = c0 * (dN.x * (F21 * S11 + F22 * S12) + dN.y * (F22 * S22 + F21 * S12));
            s_p[E(k)] = q;
        }
    }
}

// Gauss-point pass of the mixed-precision form: dN pairs stored in FP32, strain, stress and the
// contributions computed in FP32 (with fused multiply-adds), displacements gathered in FP32 as
// differences to the body's first node (taken in FP64: sum_j dN_j = 0, so the body's rigid
// translation cancels exactly and does not eat the FP32 mantissa).  Nodal force sums stay FP64.
__device__ __forceinline__ void chunk_points_mx(int t, int ngp, int mtype, float Mu, float Lam, const float2* s_upf,
                                                float2* s_p, const uint16_t* s_idx, const double* s_c0,
                                                const unsigned* s_gpm, const uint16_t* s_roff)
{
    const mel_rows R = point_rows(t, ngp, s_gpm, s_roff);
    const int ns = R.ns;
    const float c0 = (float)s_c0[t];
    if (mtype == MEL_MAT_ELASTIC_LINEAR) {
        float E11 = 0.f, E12 = 0.f, E22 = 0.f;
        int k = 0;
        for (; k + 8 <= ns; k += 8) {
            float2 dN[8], u[8];
#pragma unroll
            for (int j = 0; j < 8; j++) { const int e = E(k + j); dN[j] = s_p[e]; u[j] = s_upf[s_idx[e]]; }
#pragma unroll
            for (int j = 0; j < 8; j++) {
                E11 = __fmaf_rn(dN[j].x, u[j].x, E11);
                E12 = __fmaf_rn(dN[j].x, u[j].y, __fmaf_rn(dN[j].y, u[j].x, E12));
                E22 = __fmaf_rn(dN[j].y, u[j].y, E22);
            }
        }
        if (k < ns) {
            float2 dN[8], u[8];
#pragma unroll
            for (int j = 0; j < 8; j++)
                if (k + j < ns) { const int e = E(k + j); dN[j] = s_p[e]; u[j] = s_upf[s_idx[e]]; }
#pragma unroll
            for (int j = 0; j < 8; j++)
                if (k + j < ns) {
                    E11 = __fmaf_rn(dN[j].x, u[j].x, E11);
                    E12 = __fmaf_rn(dN[j].x, u[j].y, __fmaf_rn(dN[j].y, u[j].x, E12));
                    E22 = __fmaf_rn(dN[j].y, u[j].y, E22);
                }
        }
        E12 = 0.5f * E12;
        const float S33 = Lam * (E11 + E22);      // Apply_Elastic_Linear (Code/Model.h:19-29), J - 1 = tr E
        const float Mu2 = 2.f * Mu;
        const float S11 = __fmaf_rn(Mu2, E11, S33), S22 = __fmaf_rn(Mu2, E22, S33), S12 = Mu2 * E12;
#pragma unroll 8
        for (int k2 = 0; k2 < ns; k2++) {
            const int e = E(k2);
            const float2 dN = s_p[e];
            s_p[e] = make_float2(c0 * __fmaf_rn(dN.x, S11, dN.y * S12), c0 * __fmaf_rn(dN.y, S22, dN.x * S12));
        }
    } else {
        float G11 = 0.f, G12 = 0.f, G21 = 0.f, G22 = 0.f;   // F - I
        for (int k = 0; k < ns; k++) {
            const int e = E(k);
            const float2 dN = s_p[e];
            const float2 u = s_upf[s_idx[e]];
            G11 = __fmaf_rn(dN.x, u.x, G11); G12 = __fmaf_rn(dN.y, u.x, G12);
            G21 = __fmaf_rn(dN.x, u.y, G21); G22 = __fmaf_rn(dN.y, u.y, G22);
        }
        const float F11 = 1.f + G11, F12 = G12, F21 = G21, F22 = 1.f + G22;
        const float Kappa = Lam;                   // Apply_NeoHookean (Code/Model.h:52-73)
        const float F11F12 = F11 * F11 + F12 * F12, F21F22 = F21 * F21 + F22 * F22;
        const float Jm1 = G11 + G22 + (G11 * G22 - G12 * G21);   // J - 1 without cancellation
        const float J = 1.f + Jm1;
        const float invJ = 1.f / J;
        const float K = Kappa * Jm1;
        const float MuJ53 = Mu * powf(J, -1.666666667f);
        const float trB = 0.333333333f * (F11F12 + F21F22 + 1.f);
        const float s11 = K + MuJ53 * (F11F12 - trB), s22 = K + MuJ53 * (F21F22 - trB);
        const float s12 = MuJ53 * (F11 * F21 + F12 * F22);
        const float S11 = (F12 * (F12 * s22 - F22 * s12) - F22 * (F12 * s12 - F22 * s11)) * invJ;
        const float S22 = (F11 * (F11 * s22 - F21 * s12) - F21 * (F11 * s12 - F21 * s11)) * invJ;
        const float S12 = (F21 * (F12 * s12 - F22 * s11) - F11 * (F12 * s22 - F22 * s12)) * invJ;
        for (int k = 0; k < ns; k++) {
            const int e = E(k);
            const float2 dN = s_p[e];
            s_p[e] = make_float2(c0 * (dN.x * (F11 * S11 + F12 * S12) + dN.y * (F12 * S22 + F11 * S12)),
                                 c0 * (dN.x * (F21 * S11 + F22 * S12) + dN.y * (F22 * S22 + F21 * S12)));
        }
    }
}

#undef E

// Shared memory of a deformable body (n nodes, staging buffers of img_cap bytes each; two for the
// two-buffer loop, MEL_STAGES(1) for the pipeline):
//   s_up, s_f, s_fc        3 x n double2       displacements, internal forces, contact forces
//   s_upf (mixed only)     n2 x float2         displacements relative to node 0 (n2 = n rounded to 2)
//   ring mbarriers + abort flag                MEL_BAR_BYTES
//   region                 max(MEL_STAGES img_cap, 128 n) bytes: the ring of chunk images during
//                          the Gauss-point pass, then s_fn, s_fd, s_vp, s_ap (n double2 each), the
//                          six work terms per node (6 x n double) and, in the first half-step of
//                          Solver_step, the temporary displacement parameters (n double2)
template <bool MX, bool AD, bool WIDE>
__device__ void deformable_body(const mel_dev& d, int b, double T, double T0, char* smem)
{
    const int tid = threadIdx.x;
    const int lane = tid & 31, warp = tid >> 5;
    const int n0 = d.b_node0[b];
    const int n = d.b_node0[b + 1] - n0;
    const double dt = d.dt[0];
    // a body above MEL_MAX_BODY_NODES nodes ("wide", its own instantiation so that the others keep
    // plain shared-memory addressing) keeps its node arrays in global memory: it reads its
    // displacement parameters in place and accumulates its forces in gscr; shared memory then holds
    // only the mbarriers and the chunk images
    constexpr bool wide = WIDE;
    const long long go = WIDE ? d.b_gscr[b] : 0LL;
    double2* s_up = wide ? d.up + n0 : reinterpret_cast<double2*>(smem);
    double2* s_f = wide ? reinterpret_cast<double2*>(d.gscr + go) : s_up + n;
    double2* s_fc = s_f + n;
    float2* s_upf = reinterpret_cast<float2*>(s_fc + n);
    char* const s_after = wide ? smem : (MX ? reinterpret_cast<char*>(s_upf + ((n + 1) & ~1)) : reinterpret_cast<char*>(s_fc + n));
    // the chunk loop, which leaves the internal forces in s_f and the contact forces in s_fc
    char* region;
    volatile int* s_abort;
    // the mixed pass runs the pipeline on bodies with many chunks and the two-buffer loop on the
    // others, whose few chunks leave a three-stage pipeline mostly filling and draining
    const bool pipe = MX && d.b_pipe && d.b_pipe[b];
    if (!pipe) {
        uint64_t* s_bar = reinterpret_cast<uint64_t*>(s_after);
        s_abort = reinterpret_cast<volatile int*>(s_bar + 2);
        region = reinterpret_cast<char*>(s_bar) + MEL_BAR_BYTES;
        char* const buf0 = region;
        char* const buf1 = region + d.img_cap;
        const int ch0 = d.b_chunk0[b];
        const int nch = d.b_chunk0[b + 1] - ch0;
        for (int i = tid; i < n; i += blockDim.x) {
            if (!wide) s_up[i] = d.up[n0 + i];
            s_f[i] = make_double2(0., 0.);
            s_fc[i] = make_double2(0., 0.);
        }
        if (MX) {
            const double2 u0 = d.up[n0];
            for (int i = tid; i < n; i += blockDim.x) {
                const double2 u = d.up[n0 + i];
                s_upf[i] = make_float2((float)(u.x - u0.x), (float)(u.y - u0.y));
            }
        }
        if (tid == 0) {
            mbar_init(&s_bar[0], 1);
            mbar_init(&s_bar[1], 1);
            mbar_init_fence();
            *s_abort = 0;
        }
        __syncthreads();
        if (warp < MEL_BODY_CTHREADS / 32) {
            // ---- Update_internal_forces: chunk k is computed while chunk k+1 is in flight ----------
            const int mat = d.b_mat[b];
            const int mtype = d.mat_type[mat];
            const double Mu = d.mat_p[MEL_MAT_NPARAM * mat + 3];
            const double Lam = d.mat_p[MEL_MAT_NPARAM * mat + 4];
            int issued = 0;
            if (tid == 0)
                for (; issued < 2 && issued < nch; issued++) {
                    const mel_chunk c = d.chunk[ch0 + issued];
                    mbar_arrive_expect_tx(&s_bar[issued], (unsigned)c.bytes);
                    bulk_load(issued ? buf1 : buf0, d.img + c.img, (unsigned)c.bytes, &s_bar[issued]);
                }
            int k = 0;
            for (; k < nch; k++) {
                const int sel = k & 1;
                char* bk = sel ? buf1 : buf0;
                long long nxt_img = 0;
                int nxt_bytes = 0;
                if (tid == 0 && k + 2 < nch) { const mel_chunk c = d.chunk[ch0 + k + 2]; nxt_img = c.img; nxt_bytes = c.bytes; }
                const bool ok = mbar_wait_bounded(&s_bar[sel], (unsigned)((k >> 1) & 1), d.wait_ns);
                if (!ok) { atomicOr(&d.err[MEL_E_WAIT], 1u); *s_abort = 1; }
                const int4 hdr = ok ? *reinterpret_cast<const int4*>(bk) : make_int4(0, 0, 0, 0);
                const mel_chunk_layout L = mel_chunk_sections(hdr.x, hdr.y, hdr.z, hdr.w, MX ? 8 : 16, (!MX && wide) ? 1 : 0);
                const uint16_t* s_idx = reinterpret_cast<const uint16_t*>(bk + L.idx);
                const uint16_t* s_tpos = reinterpret_cast<const uint16_t*>(bk + L.tpos);
                const unsigned* s_tn = reinterpret_cast<const unsigned*>(bk + L.tn);
                const uint16_t* s_roff = reinterpret_cast<const uint16_t*>(bk + L.roff);
                if (tid < hdr.x) {
                    if (MX)
                        chunk_points_mx(tid, hdr.x, mtype, (float)Mu, (float)Lam, s_upf, reinterpret_cast<float2*>(bk + L.dN), s_idx,
                                        reinterpret_cast<const double*>(bk + L.c0), reinterpret_cast<const unsigned*>(bk + L.gpm),
                                        reinterpret_cast<const uint16_t*>(bk + L.roff));
                    else
                        chunk_points(tid, hdr.x, mtype, Mu, Lam, s_up, reinterpret_cast<double2*>(bk + L.dN), s_idx,
                                     reinterpret_cast<const double*>(bk + L.c0), reinterpret_cast<const unsigned*>(bk + L.gpm),
                                     reinterpret_cast<const uint16_t*>(bk + L.roff));
                }
                compute_sync();
                if (*s_abort) break;
                if (MX) {
                    // pull of the mixed form, a two-level segmented reduction in place of the ordered
                    // chains: each lane sums one piece (at most MEL_PIECE entries of one node) in FP64,
                    // then the pieces of a node, on consecutive lanes, are combined by a Hillis-Steele
                    // scan over warp shuffles (equal node keys 2^i lanes apart mean one segment, as
                    // keys are sorted) and the last lane of each segment subtracts the sum from the
                    // node.  Warp w owns the pieces [wr[w], wr[w+1]), whole nodes only, balanced by
                    // entries, so no two warps touch one node.
                    const float2* s_q = reinterpret_cast<const float2*>(bk + L.dN);
                    const uint16_t* s_wr = reinterpret_cast<const uint16_t*>(bk + L.tn);
                    const unsigned* s_pc = reinterpret_cast<const unsigned*>(bk + L.tn + 16);
                    const int p1 = s_wr[warp + 1];
                    for (int p0 = s_wr[warp]; p0 < p1; p0 += 32) {
                        const int pi = p0 + lane;
                        const bool v = pi < p1;
                        const unsigned rec = v ? s_pc[pi] : 0u;
                        const int node = v ? (int)((rec >> 16) & 0xffffu) : -1;
                        const int q0 = (int)(rec & 0x1fffu), cnt = v ? (int)((rec >> 13) & 7u) + 1 : 0;
                        float2 c[MEL_PIECE];
#pragma unroll
                        for (int i = 0; i < MEL_PIECE; i++) c[i] = i < cnt ? s_q[s_tpos[q0 + i]] : make_float2(0.f, 0.f);
                        double fx = 0., fy = 0.;
#pragma unroll
                        for (int i = 0; i < MEL_PIECE; i++) { fx = fx + (double)c[i].x; fy = fy + (double)c[i].y; }
#pragma unroll
                        for (int dd = 1; dd < 32; dd <<= 1) {
                            const double ox = __shfl_up_sync(0xffffffffu, fx, dd);
                            const double oy = __shfl_up_sync(0xffffffffu, fy, dd);
                            const int on = __shfl_up_sync(0xffffffffu, node, dd);
                            if (lane >= dd && on == node) { fx = fx + ox; fy = fy + oy; }
                        }
                        const int nn = __shfl_down_sync(0xffffffffu, node, 1);
                        if (v && (lane == 31 || nn != node)) {
                            double2 f = s_f[node];
                            f.x = f.x - fx;
                            f.y = f.y - fy;
                            s_f[node] = f;
                        }
                        __syncwarp();     // a node continued by the next round reads this update
                    }
                } else {
                    // pull: each touched node subtracts its contributions in ascending Gauss-point order.
                    // Pull slot t is lane t & 31 of group t >> 5, its entry j at row j of the group's row
                    // table.  Groups are sorted by entry count; warp w takes groups w, 13 - w, 14 + w, ...
                    // (snake order), so the heaviest group has a warp to itself and the lighter ones pair up.
                    const int ngrp = (hdr.z + 31) >> 5;
                    for (int i = 0; 7 * i < ngrp; i++) {
                        const int t = (7 * i + ((i & 1) ? 6 - warp : warp)) * 32 + lane;
                        if (t >= hdr.z) continue;
                        const unsigned rec = s_tn[t];
                        const int node = wide ? (int)reinterpret_cast<const uint16_t*>(bk + L.tnode)[t] : (int)(rec & 0xfffu);
                        const int cnt = (int)((rec >> 12) & 0xffu);
                        const uint16_t* prow = s_roff + (rec >> 20);
                        // rows every slot of a full group has: 32 wide and contiguous
                        const int pfull = (t | 31) < hdr.z ? (int)((s_tn[t | 31] >> 12) & 0xffu) : 0;
                        const int pbase = prow[0];
        #define PQ(j) ((j) < pfull ? pbase + 32 * (j) + lane : prow[(j)] + lane)
                        double2 f = s_f[node];
                        int j = 0;
                        const double2* s_p = reinterpret_cast<const double2*>(bk + L.dN);
                        for (; j + 8 <= pfull; j += 8) {
                            double2 c[8];
#pragma unroll
                            for (int i = 0; i < 8; i++) c[i] = s_p[s_tpos[pbase + 32 * (j + i) + lane]];
#pragma unroll
                            for (int i = 0; i < 8; i++) { f.x = f.x - c[i].x; f.y = f.y - c[i].y; }
                        }
                        for (; j + 8 <= cnt; j += 8) {      // remaining rows: row-table loads issued together
                            int q[8];
#pragma unroll
                            for (int i = 0; i < 8; i++) q[i] = PQ(j + i);
                            double2 c[8];
#pragma unroll
                            for (int i = 0; i < 8; i++) c[i] = s_p[s_tpos[q[i]]];
#pragma unroll
                            for (int i = 0; i < 8; i++) { f.x = f.x - c[i].x; f.y = f.y - c[i].y; }
                        }
                        for (; j + 4 <= cnt; j += 4) {
                            double2 c[4];
#pragma unroll
                            for (int i = 0; i < 4; i++) c[i] = s_p[s_tpos[PQ(j + i)]];
#pragma unroll
                            for (int i = 0; i < 4; i++) { f.x = f.x - c[i].x; f.y = f.y - c[i].y; }
                        }
                        for (; j < cnt; j++) {
                            const double2 c = s_p[s_tpos[PQ(j)]];
                            f.x = f.x - c.x;
                            f.y = f.y - c.y;
                        }
        #undef PQ
                        s_f[node] = f;
                    }
                }
                fence_proxy_async();
                compute_sync();
                if (tid == 0 && k + 2 < nch) {
                    mbar_arrive_expect_tx(&s_bar[sel], (unsigned)nxt_bytes);
                    bulk_load(bk, d.img + nxt_img, (unsigned)nxt_bytes, &s_bar[sel]);
                    issued++;
                }
            }
            if (tid == 0 && *s_abort)   // give the copies still in flight a bounded time to land
                for (int c = k; c < issued; c++) mbar_wait_bounded(&s_bar[c & 1], (unsigned)((c >> 1) & 1));
        } else {
            // ---- contact forces (warp 7): slave scatter in list order, then master scatter in send
            // order (Body::Update_contact_forces, Code/Body.h:1642-1900) ---------------------------
            for (int c = d.b_cont0[b]; c < d.b_cont0[b + 1]; c++) {
                const mel_contact* ct = d.cont + c;
                if (d.table[d.b_mat[b] * d.nmat + d.b_mat[ct->bodyM]] <= -1) continue;
                double Fsx = ct->fx, Fsy = ct->fy;
                warp_scatter(d, n0, ct->nodeS, Fsx, Fsy, s_fc, lane);
                __syncwarp();
            }
            for (int r = d.b_inc0[b]; r < d.b_inc0[b + 1]; r++) {
                int2 rg = d.inc_rng[r];
                for (int c = rg.x; c < rg.y; c++) {
                    const mel_contact* ct = d.cont + c;
                    if (d.table[d.b_mat[ct->bodyS] * d.nmat + d.b_mat[b]] <= -1) continue;
                    double Fsx = ct->fx, Fsy = ct->fy;
                    for (int k = 0; k < 4; k++) {
                        double sk = ct->shapeM[k];
                        warp_scatter(d, n0, ct->nodeM[k], -Fsx * sk, -Fsy * sk, s_fc, lane);
                        __syncwarp();
                    }
                }
            }
        }
        __syncthreads();
        if (*s_abort) return;
    } else {
        constexpr int NS = MEL_STAGES(1);
        uint64_t* s_bar = reinterpret_cast<uint64_t*>(s_after);
        // stage s of the ring: full[s] (the bulk copy landed), pointed[s] (every point thread has
        // written its contributions), empty[s] (every pull thread is done with the buffer)
        uint64_t* full = s_bar;
        uint64_t* pointed = s_bar + NS;
        uint64_t* empty = s_bar + 2 * NS;
        s_abort = reinterpret_cast<volatile int*>(s_bar + 3 * NS);
        region = reinterpret_cast<char*>(s_bar) + MEL_BAR_BYTES;
        constexpr int PTW = MEL_PT_WARPS_MX;                  // point warps 0 .. PTW-1
        constexpr int PLW = 7 - PTW;                          // pull warps PTW .. 6; warp 7 copies and scatters
        const int ch0 = d.b_chunk0[b];
        const int nch = d.b_chunk0[b + 1] - ch0;
        for (int i = tid; i < n; i += blockDim.x) {
            s_up[i] = d.up[n0 + i];
            s_f[i] = make_double2(0., 0.);
            s_fc[i] = make_double2(0., 0.);
        }
        if (MX) {
            const double2 u0 = d.up[n0];
            for (int i = tid; i < n; i += blockDim.x) {
                const double2 u = d.up[n0 + i];
                s_upf[i] = make_float2((float)(u.x - u0.x), (float)(u.y - u0.y));
            }
        }
        if (tid == 0) {
            for (int st = 0; st < NS; st++) {
                mbar_init(&full[st], 1);
                mbar_init(&pointed[st], 32 * PTW);
                mbar_init(&empty[st], 32 * PLW);
            }
            mbar_init_fence();
            *s_abort = 0;
        }
        __syncthreads();
        // ---- Update_internal_forces as a pipeline over the body's chunks: warp 7 streams chunk images
        // into a ring of NS buffers, the point warps form strain, stress and contributions of
        // chunk k while the pull warps add those of chunk k-1 to the nodes (in ascending point order,
        // chunk after chunk), so the two ordered chains and the copies overlap --------------------------
        const int mat = d.b_mat[b];
        const int mtype = d.mat_type[mat];
        const double Mu = d.mat_p[MEL_MAT_NPARAM * mat + 3];
        const double Lam = d.mat_p[MEL_MAT_NPARAM * mat + 4];
        if (warp < PTW) {
            for (int k = 0; k < nch; k++) {
                const int st = k % NS;
                char* bk = region + st * d.img_cap;
                if (*s_abort) break;
                if (!mbar_wait_bounded(&full[st], (unsigned)((k / NS) & 1), d.wait_ns)) {
                    atomicOr(&d.err[MEL_E_WAIT], 1u);
                    *s_abort = 1;
                    break;
                }
                const int4 hdr = *reinterpret_cast<const int4*>(bk);
                const mel_chunk_layout L = mel_chunk_sections(hdr.x, hdr.y, hdr.z, hdr.w, MX ? 8 : 16);
                if (tid < hdr.x) {
                    if (MX)
                        chunk_points_mx(tid, hdr.x, mtype, (float)Mu, (float)Lam, s_upf, reinterpret_cast<float2*>(bk + L.dN),
                                        reinterpret_cast<const uint16_t*>(bk + L.idx), reinterpret_cast<const double*>(bk + L.c0),
                                        reinterpret_cast<const unsigned*>(bk + L.gpm), reinterpret_cast<const uint16_t*>(bk + L.roff));
                    else
                        chunk_points(tid, hdr.x, mtype, Mu, Lam, s_up, reinterpret_cast<double2*>(bk + L.dN),
                                     reinterpret_cast<const uint16_t*>(bk + L.idx), reinterpret_cast<const double*>(bk + L.c0),
                                     reinterpret_cast<const unsigned*>(bk + L.gpm), reinterpret_cast<const uint16_t*>(bk + L.roff));
                }
                fence_proxy_async();      // these generic writes precede the copy that will refill the buffer
                mbar_arrive(&pointed[st]);
            }
        } else if (warp < 7) {
            // pull: each touched node subtracts its contributions in ascending Gauss-point order (the
            // mixed form adds its FP32 contributions in FP64).  Pull slot t is lane t & 31 of group
            // t >> 5, its entry j at row j of the group's row table.  Groups are sorted by entry count;
            // pull warp w takes groups w, 2 PLW - 1 - w, 2 PLW + w, ... (snake order).  The group's
            // barrier at the top of every chunk keeps a node's chunks in order when different warps
            // hold it, and makes the group leave together when a wait gives up.
            const int w = warp - PTW;
            for (int k = 0; k < nch; k++) {
                const int st = k % NS;
                char* bk = region + st * d.img_cap;
                const bool ok = !*s_abort && mbar_wait_bounded(&pointed[st], (unsigned)((k / NS) & 1), d.wait_ns);
                if (!ok && !*s_abort) { atomicOr(&d.err[MEL_E_WAIT], 1u); *s_abort = 1; }
                if (pull_group_any<32 * PLW>(!ok)) break;
                const int4 hdr = *reinterpret_cast<const int4*>(bk);
                const mel_chunk_layout L = mel_chunk_sections(hdr.x, hdr.y, hdr.z, hdr.w, MX ? 8 : 16);
                const uint16_t* s_tpos = reinterpret_cast<const uint16_t*>(bk + L.tpos);
                const unsigned* s_tn = reinterpret_cast<const unsigned*>(bk + L.tn);
                const uint16_t* s_roff = reinterpret_cast<const uint16_t*>(bk + L.roff);
                const int ngrp = (hdr.z + 31) >> 5;
                for (int i = 0; PLW * i < ngrp; i++) {
                    const int t = (PLW * i + ((i & 1) ? PLW - 1 - w : w)) * 32 + lane;
                    if (t >= hdr.z) continue;
                    const unsigned rec = s_tn[t];
                    const int node = (int)(rec & 0xfffu);
                    const int cnt = (int)((rec >> 12) & 0xffu);
                    const uint16_t* prow = s_roff + (rec >> 20);
                    // rows every slot of a full group has: 32 wide and contiguous
                    const int pfull = (t | 31) < hdr.z ? (int)((s_tn[t | 31] >> 12) & 0xffu) : 0;
                    const int pbase = prow[0];
    #define PQ(j) ((j) < pfull ? pbase + 32 * (j) + lane : prow[(j)] + lane)
                    double2 f = s_f[node];
                    int j = 0;
                    if (MX) {
                        const float2* s_q = reinterpret_cast<const float2*>(bk + L.dN);
                        for (; j + 8 <= pfull; j += 8) {
                            float2 c[8];
    #pragma unroll
                            for (int i = 0; i < 8; i++) c[i] = s_q[s_tpos[pbase + 32 * (j + i) + lane]];
    #pragma unroll
                            for (int i = 0; i < 8; i++) { f.x = f.x - (double)c[i].x; f.y = f.y - (double)c[i].y; }
                        }
                        for (; j + 8 <= cnt; j += 8) {      // remaining rows: row-table loads issued together
                            int q[8];
    #pragma unroll
                            for (int i = 0; i < 8; i++) q[i] = PQ(j + i);
                            float2 c[8];
    #pragma unroll
                            for (int i = 0; i < 8; i++) c[i] = s_q[s_tpos[q[i]]];
    #pragma unroll
                            for (int i = 0; i < 8; i++) { f.x = f.x - (double)c[i].x; f.y = f.y - (double)c[i].y; }
                        }
                        for (; j + 4 <= cnt; j += 4) {
                            float2 c[4];
    #pragma unroll
                            for (int i = 0; i < 4; i++) c[i] = s_q[s_tpos[PQ(j + i)]];
    #pragma unroll
                            for (int i = 0; i < 4; i++) { f.x = f.x - (double)c[i].x; f.y = f.y - (double)c[i].y; }
                        }
                        for (; j < cnt; j++) {
                            const float2 c = s_q[s_tpos[PQ(j)]];
                            f.x = f.x - (double)c.x;
                            f.y = f.y - (double)c.y;
                        }
                    } else {
                        const double2* s_p = reinterpret_cast<const double2*>(bk + L.dN);
                        for (; j + 8 <= pfull; j += 8) {
                            double2 c[8];
    #pragma unroll
                            for (int i = 0; i < 8; i++) c[i] = s_p[s_tpos[pbase + 32 * (j + i) + lane]];
    #pragma unroll
                            for (int i = 0; i < 8; i++) { f.x = f.x - c[i].x; f.y = f.y - c[i].y; }
                        }
                        for (; j + 8 <= cnt; j += 8) {      // remaining rows: row-table loads issued together
                            int q[8];
    #pragma unroll
                            for (int i = 0; i < 8; i++) q[i] = PQ(j + i);
                            double2 c[8];
    #pragma unroll
                            for (int i = 0; i < 8; i++) c[i] = s_p[s_tpos[q[i]]];
    #pragma unroll
                            for (int i = 0; i < 8; i++) { f.x = f.x - c[i].x; f.y = f.y - c[i].y; }
                        }
                        for (; j + 4 <= cnt; j += 4) {
                            double2 c[4];
    #pragma unroll
                            for (int i = 0; i < 4; i++) c[i] = s_p[s_tpos[PQ(j + i)]];
    #pragma unroll
                            for (int i = 0; i < 4; i++) { f.x = f.x - c[i].x; f.y = f.y - c[i].y; }
                        }
                        for (; j < cnt; j++) {
                            const double2 c = s_p[s_tpos[PQ(j)]];
                            f.x = f.x - c.x;
                            f.y = f.y - c.y;
                        }
                    }
    #undef PQ
                    s_f[node] = f;
                }
                fence_proxy_async();
                mbar_arrive(&empty[st]);
            }
        } else if (lane == 0) {
            // ---- producer: the first NS chunks at once, then each chunk into the buffer the
            // pull warps released ----------------------------------------------------------------------
            int issued = 0;
            for (; issued < NS && issued < nch; issued++) {
                const mel_chunk c = d.chunk[ch0 + issued];
                mbar_arrive_expect_tx(&full[issued], (unsigned)c.bytes);
                bulk_load(region + issued * d.img_cap, d.img + c.img, (unsigned)c.bytes, &full[issued]);
            }
            for (; issued < nch; issued++) {
                const int st = issued % NS;
                const mel_chunk c = d.chunk[ch0 + issued];
                if (*s_abort) break;
                if (!mbar_wait_bounded(&empty[st], (unsigned)((issued / NS - 1) & 1), d.wait_ns)) {
                    atomicOr(&d.err[MEL_E_WAIT], 1u);
                    *s_abort = 1;
                    break;
                }
                mbar_arrive_expect_tx(&full[st], (unsigned)c.bytes);
                bulk_load(region + st * d.img_cap, d.img + c.img, (unsigned)c.bytes, &full[st]);
            }
            if (*s_abort)   // give the copies still in flight a bounded time to land before the CTA ends
                for (int c = issued - 1; c >= 0 && c >= issued - NS; c--)
                    mbar_wait_bounded(&full[c % NS], (unsigned)((c / NS) & 1));
        } else {
            // ---- contact forces (lanes 1-31 of warp 7, meanwhile): slave scatter in list order, then
            // master scatter in send order (Body::Update_contact_forces, Code/Body.h:1642-1900) ---------
            const unsigned mask = 0xfffffffeu;
            for (int c = d.b_cont0[b]; c < d.b_cont0[b + 1]; c++) {
                const mel_contact* ct = d.cont + c;
                if (d.table[d.b_mat[b] * d.nmat + d.b_mat[ct->bodyM]] <= -1) continue;
                double Fsx = ct->fx, Fsy = ct->fy;
                warp_scatter(d, n0, ct->nodeS, Fsx, Fsy, s_fc, lane - 1, 31);
                __syncwarp(mask);
            }
            for (int r = d.b_inc0[b]; r < d.b_inc0[b + 1]; r++) {
                int2 rg = d.inc_rng[r];
                for (int c = rg.x; c < rg.y; c++) {
                    const mel_contact* ct = d.cont + c;
                    if (d.table[d.b_mat[ct->bodyS] * d.nmat + d.b_mat[b]] <= -1) continue;
                    double Fsx = ct->fx, Fsy = ct->fy;
                    for (int k = 0; k < 4; k++) {
                        double sk = ct->shapeM[k];
                        warp_scatter(d, n0, ct->nodeM[k], -Fsx * sk, -Fsy * sk, s_fc, lane - 1, 31);
                        __syncwarp(mask);
                    }
                }
            }
        }
        __syncwarp();
        __syncthreads();
        if (*s_abort) return;
    }
    double2* s_fn = reinterpret_cast<double2*>(wide ? d.gscr + go + mel_wide_pre_bytes(n) : region);
    double2* s_fd = s_fn + n;
    double2* s_vp = s_fd + n;
    double2* s_ap = s_vp + n;
    double* s_T = reinterpret_cast<double*>(s_ap + n);
    const int has_bc = d.b_has_bc[b];
    if (has_bc) {
        for (int i = tid; i < n; i += blockDim.x) { s_fn[i] = make_double2(0., 0.); s_fd[i] = make_double2(0., 0.); }
        __syncthreads();
        if (warp == 1) {
            // ---- Update_bc_forces, deformable (Code/Body.h:669-799) ----------------------
            for (int g = d.b_bd0[b]; g < d.b_bd0[b + 1]; g++) {
                int tx = d.bd_bc[2 * g], ty = d.bd_bc[2 * g + 1];
                if (tx == MEL_BC_NONE && ty == MEL_BC_NONE) continue;
                double xv, xvel, yv, yvel;
                border_bc_value(d, g, 0, T, xv, xvel);
                border_bc_value(d, g, 1, T, yv, yvel);
                int e0 = d.bd_e0[g], nbn = d.bd_e0[g + 1] - e0;
                for (int k = 0; k < nbn - 1; k++) {
                    int e = e0 + k;
                    int bn = d.e_node[e];
                    double length = border_length(d, b, g, k);
                    double px = 0., py = 0.;
                    double ftx = 0., fty = 0., ftpx = 0., ftpy = 0.;
                    if (tx == MEL_BC_FOLLOWING || ty == MEL_BC_FOLLOWING) {
                        int a0 = n0 + d.e_sn[4 * e], a2 = n0 + d.e_sn[4 * e + 2];
                        double2 X0 = d.X0[a0], X2 = d.X0[a2], x0 = d.x[a0], x2 = d.x[a2];
                        double invl = mel_rsqrt((X2.x - X0.x) * (X2.x - X0.x) + (X2.y - X0.y) * (X2.y - X0.y));
                        double invlp = mel_rsqrt((x2.x - x0.x) * (x2.x - x0.x) + (x2.y - x0.y) * (x2.y - x0.y));
                        ftx = (X2.x - X0.x) * invl; fty = (X2.y - X0.y) * invl;
                        ftpx = (x2.x - x0.x) * invlp; ftpy = (x2.y - x0.y) * invlp;
                    }
                    double2 ub = d.u[n0 + bn], vb = d.v[n0 + bn];
                    if (tx == MEL_BC_ORIENTED) px = xv;
                    else if (tx == MEL_BC_FOLLOWING) { px += xv * (ftx * ftpx + fty * ftpy); py += xv * (ftx * ftpy - fty * ftpx); }
                    else if (tx == MEL_BC_SOFT) px = d.bd_bcp[4 * g] * (xv - ub.x) - d.bd_bcp[4 * g + 1] * (xvel - vb.x);
                    if (ty == MEL_BC_ORIENTED) py = yv;
                    else if (ty == MEL_BC_FOLLOWING) { px += yv * (fty * ftpx - ftx * ftpy); py += yv * (fty * ftpy + ftx * ftpx); }
                    else if (ty == MEL_BC_SOFT) py = d.bd_bcp[4 * g + 2] * (yv - ub.y) - d.bd_bcp[4 * g + 3] * (yvel - vb.y);
                    if (lane == 0) d.e_bcp[e] = make_double2(px, py);   // Border::x_bc_pressure, y_bc_pressure
                    int gn = n0 + bn;
                    for (int j = d.sup_ptr[gn] + lane; j < d.sup_ptr[gn + 1]; j += 32) {
                        double sf = d.sup_N[j];
                        double fxn = 0., fyn = 0., fxd = 0., fyd = 0.;
                        if (tx == MEL_BC_ORIENTED) fxn = px * length * sf;
                        else if (tx == MEL_BC_FOLLOWING) { fxn = px * length * sf; fyn = py * length * sf; }
                        else if (tx == MEL_BC_SOFT) fxd = px * length * sf;
                        if (ty == MEL_BC_ORIENTED) fyn = py * length * sf;
                        else if (ty == MEL_BC_FOLLOWING) { fxn = px * length * sf; fyn = py * length * sf; }
                        else if (ty == MEL_BC_SOFT) fyd = py * length * sf;
                        int t = d.sup_idx[j];
                        double2 a = s_fn[t]; a.x = a.x + fxn; a.y = a.y + fyn; s_fn[t] = a;
                        double2 c = s_fd[t]; c.x = c.x + fxd; c.y = c.y + fyd; s_fd[t] = c;
                    }
                    __syncwarp();
                }
            }
        }
        __syncthreads();
    }
    // ---- Sum_up_forces, Apply_Newton (Code/Node.h:212-231); work terms of Body::Apply_Euler
    // (Code/Body.h:2058-2066) per node, summed in node order below ---------------------------
    const double gx = (d.b_status[b] == MEL_STATUS_NOGRAVITY) ? 0. : d.gx;
    const double gy = (d.b_status[b] == MEL_STATUS_NOGRAVITY) ? 0. : d.gy;
    // Apply_Euler's Deltat: the step, or half of it in each half-step of Solver_step
    const double dte = AD ? dt * 0.5 : dt;
    const double hdt = 0.5 * dte;
    double2* s_upt = reinterpret_cast<double2*>(s_T + 6 * n);     // AD phase 1: temporary parameters
    for (int i = tid; i < n; i += blockDim.x) {
        int gi = n0 + i;
        double2 m = d.mass[gi], im = d.minv[gi];
        double2 fb = make_double2(m.x * gx, m.y * gy);
        double2 fi = s_f[i], fc = s_fc[i];
        double2 fn = has_bc ? s_fn[i] : make_double2(0., 0.);
        double2 fd = has_bc ? s_fd[i] : make_double2(0., 0.);
        const double2 fdp = d.fdamp ? d.fdamp[gi] : make_double2(0., 0.);
        const double2 fal = d.falid ? d.falid[gi] : make_double2(0., 0.);
        double2 ft;
        ft.x = fi.x + fc.x + 0. + fb.x + fd.x + fn.x + fdp.x + fal.x;
        ft.y = fi.y + fc.y + 0. + fb.y + fd.y + fn.y + fdp.y + fal.y;
        double2 ap;
        if (AD) { const double2 f = d.fms[gi]; ap = make_double2(ft.x * im.x / f.x, ft.y * im.y / f.y); }
        else ap = make_double2(ft.x * im.x / 1., ft.y * im.y / 1.);
        double2 vp = d.vp[gi];
        s_ap[i] = ap;
        s_vp[i] = vp;
        if (d.record_forces) {
            d.o_fint[gi] = fi; d.o_fcon[gi] = fc; d.o_fneu[gi] = fn; d.o_fdir[gi] = fd; d.o_ftot[gi] = ft;
        }
        if (AD && d.phase == 1) {      // Apply_Euler_temporary(Deltat) (Code/Node.h:247-251)
            const double2 up = s_up[i];
            const double2 t = make_double2(up.x + dt * (vp.x + dt * ap.x), up.y + dt * (vp.y + dt * ap.y));
            s_upt[i] = t;
            d.upt[gi] = t;
        }
        double vx = vp.x + hdt * ap.x, vy = vp.y + hdt * ap.y;
        s_T[i] = dte * (vx * fi.x + vy * fi.y);
        s_T[n + i] = dte * (vx * fb.x + vy * fb.y);
        s_T[2 * n + i] = dte * (vx * fd.x + vy * fd.y);
        s_T[3 * n + i] = dte * (vx * fn.x + vy * fn.y);
        s_T[4 * n + i] = dte * (vx * fdp.x + vy * fdp.y);
        s_T[5 * n + i] = dte * (vx * fal.x + vy * fal.y);
    }
    __syncthreads();
    if (warp == 0) {
        // works (internal, body, dirichlet, neumann, damping, alid), summed in node order; these
        // serial sums are the body's last work for warp 0, and they overlap the kinematics below
        if (lane < 6) {
            const int w = lane == 0 ? 0 : lane + 1;       // works slots 0, 2, 3, 4, 5, 6
            d.works[7 * b + w] = ordered_sum(d.works[7 * b + w], s_T + (size_t)lane * n, n, 1);
        }
        return;
    } else {
        // ---- Apply_Euler (Code/Node.h:239-245) ---------------------------------------------
        for (int i = tid - 32; i < n; i += blockDim.x - 32) {
            int gi = n0 + i;
            double2 ap = s_ap[i], vp = s_vp[i], up = s_up[i];
            vp.x = vp.x + dte * ap.x; vp.y = vp.y + dte * ap.y;
            up.x = up.x + dte * vp.x; up.y = up.y + dte * vp.y;
            s_vp[i] = vp; s_up[i] = up;
            d.ap[gi] = ap; d.vp[gi] = vp; d.up[gi] = up;
        }
    }
    tail_sync();      // warps 1-7: Euler done
    // ---- Update_kinematics + Update_current_positions (Code/Body.h:2176-2227, 2272-2283) --
    // slot i of the body's kinematics layout is lane i & 31 of group i >> 5 (i = tid - 32 + 224 m
    // keeps the lane); row k of a group is 32 consecutive entries, so the support loads of a warp
    // are coalesced.  Each node sums its supports in their own order.
    const int ks = d.b_ks0[b];
    for (int i = tid - 32; i < n; i += blockDim.x - 32) {
        const unsigned rec = d.ks_rec[ks + i];
        const int node = (int)(rec & 0xffffu), cnt = (int)(rec >> 16);
        const int* kb = d.kg_base + ((ks + i) >> 5);
        const uint16_t* kidx = d.ks_idx + *kb + lane;
        const double* kN = d.ks_N + *kb + lane;
        double dx = 0., dy = 0., vx = 0., vy = 0., ax = 0., ay = 0.;
        int k = 0;
        for (; k + 4 <= cnt; k += 4) {
            int t[4];
            double sN[4];
#pragma unroll
            for (int q = 0; q < 4; q++) { t[q] = kidx[32 * (k + q)]; sN[q] = kN[32 * (k + q)]; }
#pragma unroll
            for (int q = 0; q < 4; q++) {
                double2 up = s_up[t[q]], vp = s_vp[t[q]], ap = s_ap[t[q]];
                double sv = sN[q];
                dx += sv * up.x; dy += sv * up.y;
                vx += sv * vp.x; vy += sv * vp.y;
                ax += sv * ap.x; ay += sv * ap.y;
            }
        }
        for (; k < cnt; k++) {
            const int t = kidx[32 * k];
            const double sv = kN[32 * k];
            double2 up = s_up[t], vp = s_vp[t], ap = s_ap[t];
            dx += sv * up.x; dy += sv * up.y;
            vx += sv * vp.x; vy += sv * vp.y;
            ax += sv * ap.x; ay += sv * ap.y;
        }
        const int gi = n0 + node;
        d.u[gi] = make_double2(dx, dy);
        d.v[gi] = make_double2(vx, vy);
        d.a[gi] = make_double2(ax, ay);
        double2 X = d.X0[gi];
        d.x[gi] = make_double2(X.x + dx, X.y + dy);
        if (AD && d.phase == 1) {      // Update_kinematics_temporary (Code/Body.h:2235-2253)
            double tx = 0., ty = 0.;
            for (int q = 0; q < cnt; q++) {
                const double2 t = s_upt[kidx[32 * q]];
                const double sv = kN[32 * q];
                tx += sv * t.x; ty += sv * t.y;
            }
            d.ut[gi] = make_double2(tx, ty);
        }
    }
    if (AD && d.phase == 2) {
        // ---- Update_bc(Time+Deltat) of the body's driven borders, Compute_error and
        // Compute_mass_scaling (Code/Body.h:2528-2594, Code/Node.h:253-320): nodal terms in
        // parallel, the body's sums and maximum in node order --------------------------------------
        double* drv = d.drv + 8 * b;
        if (tid == 32) body_drivendof(d, b, T0 + dt, drv);
        tail_sync();
        double* s_en = reinterpret_cast<double*>(s_fn);
        double* s_mms = s_en + n;
        const bool ms = d.solver == MEL_SOLVER_MASS_SCALING || d.solver == MEL_SOLVER_ADAPTIVE_MASS_SCALING;
        const double te = d.sp[0], mxs = d.sp[3], cms = d.sp[4], efac = d.sp[5], decr = d.sp[6];
        for (int i = tid - 32; i < n; i += blockDim.x - 32) {
            const int gi = n0 + i;
            const double2 u = d.u[gi], ut = d.ut[gi];
            const double ex = drv[0] == 1. ? 0. : u.x - ut.x;
            const double ey = drv[4] == 1. ? 0. : u.y - ut.y;
            const double ide = d.ide[gi];
            d.errv[gi] = make_double2(ex, ey);
            s_en[i] = sqrt(ex * ex + ey * ey) * ide;
            if (ms) {
                double2 f = d.fms[gi];
                double e[2] = { fabs(ex * ide), fabs(ey * ide) };
                double* fk[2] = { &f.x, &f.y };
                for (int k = 0; k < 2; k++) {
                    if (e[k] >= te * efac) {
                        *fk[k] += ms_pow((e[k] - te * efac), cms);
                        if (*fk[k] > mxs) *fk[k] = mxs;
                    } else {
                        if (*fk[k] != 1) *fk[k] *= decr;
                        if (*fk[k] < 1) *fk[k] = 1;
                    }
                }
                d.fms[gi] = f;
                const double2 m = d.mass[gi];
                s_mms[i] = sqrt(m.x * m.x * f.x * f.x + m.y * m.y * f.y * f.y);
            }
        }
        tail_sync();
        if (tid == 32) {
            double tot = 0., mx = 0., mm = 0.;
            for (int i = 0; i < n; i++) {
                const double en = s_en[i];
                tot += en;
                const double e2 = en == 0. ? 1.e-16 : en;
                if (e2 > mx) mx = e2;
                if (ms) mm += s_mms[i];
            }
            d.terr[b] = tot;
            d.merr[b] = mx;
            d.bmms[b] = mm;
        }
    }
}

// ------------------------------------------------------------------------------------------
// body kernel: rigid path
// ------------------------------------------------------------------------------------------
#define MEL_RIGID_BATCH 512   // border entries whose terms are staged at once (6 doubles each)

template <bool AD>
__device__ void rigid_body(const mel_dev& d, int b, double T, double T0, char* smem)
{
    const int tid = threadIdx.x;
    const int n0 = d.b_node0[b];
    const int n = d.b_node0[b + 1] - n0;
    const double dt = d.dt[0];
    double* rg = d.rg + MEL_RIGID_NF * b;
    double* rf = d.rf + 15 * b;
    double* sh = reinterpret_cast<double*>(smem);   // [0..14] forces, [16..23] drivendof, [24..32] sums
    double* sT = sh + 64;                            // staged border terms, 6 x MEL_RIGID_BATCH
    const double xcs = rg[MEL_RG_XC], ycs = rg[MEL_RG_YC];   // centre at the start of the step
    // ---- Update_bc_forces, rigid (Code/Body.h:800-899): terms of every border entry computed in
    // parallel, then each of the six sums (Neumann x, y, moment; Dirichlet x, y, moment) added
    // in entry order by one lane.  Borders whose conditions are all none or driven add only zero
    // terms (+0 leaves the sums unchanged for finite positions) and are skipped. -----------------
    double acc = 0.;                                   // lane k < 6 of warp 0: sum k
    for (int g = d.b_bd0[b]; g < d.b_bd0[b + 1]; g++) {
        int tx = d.bd_bc[2 * g], ty = d.bd_bc[2 * g + 1];
        bool activex = tx == MEL_BC_ORIENTED || tx == MEL_BC_FOLLOWING || tx == MEL_BC_SOFT;
        bool activey = ty == MEL_BC_ORIENTED || ty == MEL_BC_FOLLOWING || ty == MEL_BC_SOFT;
        if (!activex && !activey) continue;
        double xv, xvel, yv, yvel;
        border_bc_value(d, g, 0, T, xv, xvel);
        border_bc_value(d, g, 1, T, yv, yvel);
        for (int e0 = d.bd_e0[g]; e0 < d.bd_e0[g + 1]; e0 += MEL_RIGID_BATCH) {
            int ne = min(MEL_RIGID_BATCH, d.bd_e0[g + 1] - e0);
            for (int i = tid; i < ne; i += blockDim.x) {
                int e = e0 + i;
                int gn = n0 + d.e_node[e];
                double length = d.e_len0[e];
                double fxn = 0., fyn = 0., fxd = 0., fyd = 0.;
                double2 ub = d.u[gn], vb = d.v[gn], xb = d.x[gn];
                double px = 0., py = 0.;                  // Border::x_bc_pressure, y_bc_pressure
                if (tx == MEL_BC_ORIENTED || tx == MEL_BC_FOLLOWING) { px = xv; fxn = px * length; }
                else if (tx == MEL_BC_SOFT) { px = d.bd_bcp[4 * g] * (xv - ub.x) + d.bd_bcp[4 * g + 1] * (xvel - vb.x); fxd = px * length; }
                if (ty == MEL_BC_ORIENTED || ty == MEL_BC_FOLLOWING) { py = yv; fyn = py * length; }
                else if (ty == MEL_BC_SOFT) { py = d.bd_bcp[4 * g + 2] * (yv - ub.y) + d.bd_bcp[4 * g + 3] * (yvel - vb.y); fyd = py * length; }
                d.e_bcp[e] = make_double2(px, py);
                double dx = xb.x - xcs, dy = xb.y - ycs;
                sT[i] = fxn;
                sT[MEL_RIGID_BATCH + i] = fyn;
                sT[2 * MEL_RIGID_BATCH + i] = -fxn * dy + fyn * dx;
                sT[3 * MEL_RIGID_BATCH + i] = fxd;
                sT[4 * MEL_RIGID_BATCH + i] = fyd;
                sT[5 * MEL_RIGID_BATCH + i] = -fxd * dy + fyd * dx;
            }
            __syncthreads();
            if (tid < 6) acc = ordered_sum(acc, sT + tid * MEL_RIGID_BATCH, ne, 1);
            __syncthreads();
        }
    }
    // ---- contact forces: own contacts in list order (Code/Body.h:1866-1877), then the incoming
    // ranges in send order; lanes 8..10 of warp 0 each carry one of the three sums -------------
    if (tid >= 8 && tid < 11) {
        const int k = tid - 8;
        double con = 0.;
        int c0 = d.b_cont0[b], c1 = d.b_cont0[b + 1];
        con = ordered_sum(con, d.cont_rt + 6 * (size_t)c0 + k, c1 - c0, 6);
        for (int r = d.b_inc0[b]; r < d.b_inc0[b + 1]; r++) {
            int2 rr = d.inc_rng[r];
            con = ordered_sum(con, d.cont_rt + 6 * (size_t)rr.x + 3 + k, rr.y - rr.x, 6);
        }
        sh[24 + 6 + k] = con;
    }
    if (tid < 6) sh[24 + tid] = acc;
    __syncthreads();
    if (tid == 0) {
        const double neu[3] = { sh[24], sh[25], sh[26] }, dir[3] = { sh[27], sh[28], sh[29] };
        const double con[3] = { sh[30], sh[31], sh[32] };
        // Update_body_forces (Code/Body.h:925-928)
        double gx = (d.b_status[b] == MEL_STATUS_NOGRAVITY) ? 0. : d.gx;
        double gy = (d.b_status[b] == MEL_STATUS_NOGRAVITY) ? 0. : d.gy;
        double body[3] = { rg[MEL_RG_MASS] * gx, rg[MEL_RG_MASS] * gy, rf[5] };
        for (int k = 0; k < 3; k++) { rf[k] = con[k]; rf[3 + k] = body[k]; rf[6 + k] = dir[k]; rf[9 + k] = neu[k]; }
        // Sum_up_forces (Code/Body.h:1996-1998), Apply_Newton (Code/Body.h:2034-2036)
        double tot[3];
        for (int k = 0; k < 3; k++) tot[k] = rf[k] + rf[3 + k] + rf[6 + k] + rf[9 + k] + rf[12 + k];
        for (int k = 0; k < 3; k++) d.rtot[3 * b + k] = tot[k];
        const double fmsb = AD ? d.bfms[b] : 1.;
        rg[MEL_RG_XA] = tot[0] * rg[MEL_RG_INV_MASS] / fmsb;
        rg[MEL_RG_YA] = tot[1] * rg[MEL_RG_INV_MASS] / fmsb;
        rg[MEL_RG_RA] = tot[2] * rg[MEL_RG_INV_INERTIA] / fmsb;
        sh[0] = rg[MEL_RG_XA]; sh[1] = rg[MEL_RG_YA];
        // nodal copies of the body forces made by Body::Sum_up_forces (Code/Body.h:2000-2013)
        for (int k = 0; k < 3; k++) sh[2 + k] = rf[k];
        for (int k = 0; k < 3; k++) sh[5 + k] = rf[6 + k];
        for (int k = 0; k < 3; k++) sh[8 + k] = rf[9 + k];
        for (int k = 0; k < 3; k++) sh[11 + k] = tot[k];
        // Update_bc(t+dt) (Code/Body.h:335-395); the first half-step of Solver_step keeps the
        // values of the last call
        double* drv = d.drv + 8 * b;
        if (!AD) body_drivendof(d, b, T + dt, drv);
        else if (d.phase == 2) body_drivendof(d, b, T0 + dt, drv);
        const double dte = AD ? dt * 0.5 : dt;        // Apply_Euler's Deltat
        if (AD && d.phase == 1) {
            // Apply_Euler_temporary(Deltat), rigid (Code/Body.h:2133-2167)
            double* tm = d.rg_tmp + 6 * b;
            if (drv[0] == 0.) { tm[3] = rg[MEL_RG_XV] + dt * rg[MEL_RG_XA]; tm[0] = rg[MEL_RG_XD] + dt * tm[3]; }
            else if (drv[0] == 1.) { tm[3] = drv[2]; tm[0] = drv[1]; }
            if (drv[4] == 0.) { tm[4] = rg[MEL_RG_YV] + dt * rg[MEL_RG_YA]; tm[1] = rg[MEL_RG_YD] + dt * tm[4]; }
            else if (drv[4] == 1.) { tm[4] = drv[6]; tm[1] = drv[5]; }
            if (drv[0] == 0. && drv[4] == 0. && !d.b_per[b]) { tm[5] = rg[MEL_RG_RV] + dt * rg[MEL_RG_RA]; tm[2] = rg[MEL_RG_RD] + dt * tm[5]; }
            else { tm[5] = 0.; tm[2] = 0.; }
        }
        // Apply_Euler, rigid (Code/Body.h:2071-2117)
        double* W = d.works + 7 * b;
        double vx = rg[MEL_RG_XV] + 0.5 * dte * rg[MEL_RG_XA];
        double vy = rg[MEL_RG_YV] + 0.5 * dte * rg[MEL_RG_YA];
        double vr = rg[MEL_RG_RV] + 0.5 * dte * rg[MEL_RG_RA];
        W[2] += dte * (vx * rf[3] + vy * rf[4] + vr * rf[5]);
        W[3] += dte * (vx * rf[6] + vy * rf[7] + vr * rf[8]);
        W[4] += dte * (vx * rf[9] + vy * rf[10] + vr * rf[11]);
        W[5] += dte * (vx * rf[12] + vy * rf[13] + vr * rf[14]);
        if (drv[0] == 0.) { rg[MEL_RG_XV] += dte * rg[MEL_RG_XA]; rg[MEL_RG_XD] = rg[MEL_RG_XD] + dte * rg[MEL_RG_XV]; }
        else if (drv[0] == 1.) { rg[MEL_RG_XA] = drv[3]; rg[MEL_RG_XV] = drv[2]; rg[MEL_RG_XD] = drv[1]; rf[6] = rg[MEL_RG_MASS] * rg[MEL_RG_XA] - tot[0]; }
        if (drv[4] == 0.) { rg[MEL_RG_YV] += dte * rg[MEL_RG_YA]; rg[MEL_RG_YD] = rg[MEL_RG_YD] + dte * rg[MEL_RG_YV]; }
        else if (drv[4] == 1.) { rg[MEL_RG_YA] = drv[7]; rg[MEL_RG_YV] = drv[6]; rg[MEL_RG_YD] = drv[5]; rf[7] = rg[MEL_RG_MASS] * rg[MEL_RG_YA] - tot[1]; }
        if (drv[0] == 0. && drv[4] == 0. && !d.b_per[b]) { rg[MEL_RG_RV] += dte * rg[MEL_RG_RA]; rg[MEL_RG_RD] = rg[MEL_RG_RD] + dte * rg[MEL_RG_RV]; }
        else { rg[MEL_RG_RV] = 0.; rg[MEL_RG_RD] = 0.; }
        rg[MEL_RG_XC] = rg[MEL_RG_X0] + rg[MEL_RG_XD];
        rg[MEL_RG_YC] = rg[MEL_RG_Y0] + rg[MEL_RG_YD];
        rg[MEL_RG_RC] = rg[MEL_RG_R0] + rg[MEL_RG_RD];
        if (AD && d.phase == 2) {
            // Compute_error and Compute_mass_scaling, rigid (Code/Body.h:2538-2552, 2572-2593)
            const double* tm = d.rg_tmp + 6 * b;
            double te2 = 0.;
            if (drv[0] != 1.) te2 += (rg[MEL_RG_XD] - tm[0]) * (rg[MEL_RG_XD] - tm[0]);
            if (drv[4] != 1.) te2 += (rg[MEL_RG_YD] - tm[1]) * (rg[MEL_RG_YD] - tm[1]);
            te2 = 0.1 * sqrt(te2) / d.b_dist[3 * b];
            if (te2 == 0.) te2 = 1.e-16;
            d.terr[b] = te2;
            d.merr[b] = te2;
            if (d.solver == MEL_SOLVER_MASS_SCALING || d.solver == MEL_SOLVER_ADAPTIVE_MASS_SCALING) {
                const double te = d.sp[0], mxs = d.sp[3], cms = d.sp[4], efac = d.sp[5], decr = d.sp[6];
                double f = d.bfms[b];
                if (te2 >= te * efac) {
                    d.bdfms[b] = ms_pow((te2 - te * efac), cms);
                    f += d.bdfms[b];
                    if (f >= mxs) f = mxs;
                } else {
                    if (f != 1) f *= decr;
                    if (f < 1) f = 1;
                }
                d.bfms[b] = f;
                d.bmms[b] = rg[MEL_RG_MASS] * f;
            }
        }
    }
    __syncthreads();
    // node kinematics (Code/Body.h:2212-2225, 2284-2300); Apply_Newton's nodal accelerations
    const double ax = sh[0], ay = sh[1];
    const double xc = rg[MEL_RG_XC], yc = rg[MEL_RG_YC];
    const double xd = rg[MEL_RG_XD], yd = rg[MEL_RG_YD], rd = rg[MEL_RG_RD];
    const double xvb = rg[MEL_RG_XV], yvb = rg[MEL_RG_YV], rv = rg[MEL_RG_RV];
    const double x0 = rg[MEL_RG_X0], y0 = rg[MEL_RG_Y0], r0 = rg[MEL_RG_R0];
    const double dr = rd - r0;
    const double cr = mel_cos(dr), sr = mel_sin(dr);   // correctly rounded (mel_sincos.h)
    for (int i = tid; i < n; i += blockDim.x) {
        int gi = n0 + i;
        double2 X = d.X0[gi];
        double dx = X.x - x0, dy = X.y - y0;
        d.u[gi] = make_double2(xd + dx * cr - dy * sr - dx, yd + dx * sr + dy * cr - dy);
        double2 xn = make_double2(xc + dx * cr - dy * sr, yc + dx * sr + dy * cr);
        d.x[gi] = xn;
        double ddx = xn.x - xc, ddy = xn.y - yc;
        d.v[gi] = make_double2(-ddy * rv + xvb, ddx * rv + yvb);
        d.a[gi] = make_double2(ax, ay);
        if (d.record_forces) {
            d.o_fint[gi] = make_double2(0., 0.);
            d.o_fcon[gi] = make_double2(sh[2], sh[3]);
            d.o_fdir[gi] = make_double2(sh[5], sh[6]);
            d.o_fneu[gi] = make_double2(sh[8], sh[9]);
            d.o_ftot[gi] = make_double2(sh[11], sh[12]);
        }
    }
}

// contact_work of body b: the reference adds 0.5*W to the slave body and to the master body while
// looping over bodies in index order (Code/Body.h:1847-1848); incoming ranges are in that order.
__device__ void contact_work(const mel_dev& d, int b)
{
    double w = d.works[7 * b + 1];
    bool own_done = false;
    for (int r = d.b_inc0[b]; r <= d.b_inc0[b + 1]; r++) {
        bool last = (r == d.b_inc0[b + 1]);
        int2 rr = last ? make_int2(0, 0) : d.inc_rng[r];
        if (!last && rr.x == rr.y) continue;                      // empty range: nothing to read
        int sender = last ? d.nb : d.cont[rr.x].bodyS;
        if (!own_done && sender >= b) {
            for (int c = d.b_cont0[b]; c < d.b_cont0[b + 1]; c++) {
                double h = 0.5 * d.cont_w[c];
                w += h;
                if (d.cont[c].bodyM == b) w += h;
            }
            own_done = true;
        }
        if (last) break;
        if (sender == b) continue;                                // self contacts were added above
        for (int c = rr.x; c < rr.y; c++) w += 0.5 * d.cont_w[c];
    }
    d.works[7 * b + 1] = w;
}

template <bool MX, bool AD = false>
__device__ __forceinline__ void body_cta(const mel_dev& d, int bb, double T, char* smem, double T0 = 0.)
{
    int b = d.b_order[bb];
    if (d.b_status[b] == MEL_STATUS_INACTIVE) return;
    if (d.any_damped && threadIdx.x == 32) contact_work(d, b);
    if (d.b_type[b] == MEL_BODY_RIGID) rigid_body<AD>(d, b, T, T0, smem);
    else deformable_body<MX, AD, false>(d, b, T, T0, smem);
}

// bodies above MEL_MAX_BODY_NODES nodes, ordered last in b_order, run in a launch of their own so
// that their global-memory variant does not weigh on the registers of the kernel every other body
// runs
template <bool MX, bool AD = false>
__device__ __forceinline__ void wide_body_cta(const mel_dev& d, int bb, double T, char* smem, double T0 = 0.)
{
    const int b = d.b_order[bb];
    if (d.b_status[b] == MEL_STATUS_INACTIVE) return;
    if (d.any_damped && threadIdx.x == 32) contact_work(d, b);
    deformable_body<MX, AD, true>(d, b, T, T0, smem);
}

__global__ void __launch_bounds__(128) contact_kernel(mel_dev d, double law_dt_scale, int czm_init)
{
    contact_thread(d, blockIdx.x * blockDim.x + threadIdx.x, law_dt_scale, czm_init);
}

// One model: CTA i is the body d.b_order[i]; time2[parity] is the step's start time, the step's
// end time goes to time2[parity ^ 1] (the next launch reads it).
template <bool MX>
__global__ void __launch_bounds__(MEL_BODY_THREADS, 2) body_kernel(mel_dev d, int parity)
{
    extern __shared__ __align__(16) char smem[];
    const double T = d.time2[parity];
    body_cta<MX>(d, blockIdx.x, T, smem);
    if (blockIdx.x == 0 && threadIdx.x == 0) d.time2[parity ^ 1] = T + d.dt[0];
}

// One half-step of Solver_step (d.phase 1 or 2) of one model: T0 = Time, Tf = the time the
// border conditions of the forces are taken at.  The host keeps the time.
template <bool MX>
__global__ void __launch_bounds__(MEL_BODY_THREADS, 2) body_kernel_adaptive(mel_dev d, double T0, double Tf)
{
    extern __shared__ __align__(16) char smem[];
    body_cta<MX, true>(d, blockIdx.x, Tf, smem, T0);
}

// The wide bodies b_order[first + i]; the step's end time is written here when the launch above
// had no CTA (set_time)
template <bool MX>
__global__ void __launch_bounds__(MEL_BODY_THREADS, 2) body_kernel_wide(mel_dev d, int parity, int first, int set_time)
{
    extern __shared__ __align__(16) char smem[];
    const double T = d.time2[parity];
    wide_body_cta<MX>(d, first + blockIdx.x, T, smem);
    if (set_time && blockIdx.x == 0 && threadIdx.x == 0) d.time2[parity ^ 1] = T + d.dt[0];
}

template <bool MX>
__global__ void __launch_bounds__(MEL_BODY_THREADS, 2) body_kernel_adaptive_wide(mel_dev d, double T0, double Tf, int first)
{
    extern __shared__ __align__(16) char smem[];
    wide_body_cta<MX, true>(d, first + blockIdx.x, Tf, smem, T0);
}

// Solver_step's sums over bodies in body order (Code/Solver.h:289-331)
__global__ void error_reduce_kernel(mel_dev d, double* out)
{
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    double mean = 0., mx = 0., tm = 0., mm = 0.;
    int nnodes = 0;
    const bool ms = d.solver == MEL_SOLVER_MASS_SCALING || d.solver == MEL_SOLVER_ADAPTIVE_MASS_SCALING;
    for (int i = 0; i < d.nb; i++) {
        if (d.b_status[i] == MEL_STATUS_INACTIVE) continue;
        mean += d.terr[i];
        nnodes += d.b_node0[i + 1] - d.b_node0[i];
        if (d.merr[i] > mx) mx = d.merr[i];
    }
    mean /= nnodes;
    if (ms)
        for (int i = 0; i < d.nb; i++) {
            if (d.b_status[i] == MEL_STATUS_INACTIVE) continue;
            tm += d.bmms[i];
            const double inv = d.rg[MEL_RIGID_NF * i + MEL_RG_INV_MASS];
            if (d.bmms[i] * inv > mm) mm = d.bmms[i] * inv;
        }
    out[0] = mean; out[1] = mx; out[2] = tm; out[3] = mm;
}

// ---- batches: several independent models (samples) advanced by the same launches -----------
// devs[s] is the descriptor of sample s; cta0 / thr0 are prefix sums of the samples' bodies and of
// their contact-pass threads (contacts + border entries).  A sample's time lives in time2[0] and is
// advanced by advance_kernel after each step.  Every sample runs exactly the code of a one-model
// launch on its own arrays, so its results do not depend on the rest of the batch.
__device__ __forceinline__ int batch_member(const int* prefix, int nsamp, int i)
{
    int lo = 0, hi = nsamp;                  // largest s with prefix[s] <= i
    while (hi - lo > 1) { int mid = (lo + hi) >> 1; if (prefix[mid] <= i) lo = mid; else hi = mid; }
    return lo;
}

__global__ void __launch_bounds__(128) contact_kernel_batch(const mel_dev* devs, const int* thr0, int nsamp,
                                                            double law_dt_scale)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= thr0[nsamp]) return;
    const int s = batch_member(thr0, nsamp, i);
    contact_thread(devs[s], i - thr0[s], law_dt_scale);
}

template <bool MX>
__global__ void __launch_bounds__(MEL_BODY_THREADS, 2) body_kernel_batch(const mel_dev* devs, const int* cta0, int nsamp,
                                                                         int cta_base)
{
    extern __shared__ __align__(16) char smem[];
    __shared__ mel_dev sd;                   // the sample's descriptor, read once per CTA
    const int c = (int)blockIdx.x + cta_base;
    const int s = batch_member(cta0, nsamp, c);
    {
        const int* src = reinterpret_cast<const int*>(devs + s);
        int* dst = reinterpret_cast<int*>(&sd);
        for (int k = threadIdx.x; k < (int)(sizeof(mel_dev) / sizeof(int)); k += blockDim.x) dst[k] = src[k];
    }
    __syncthreads();
    body_cta<MX>(sd, c - cta0[s], sd.time2[0], smem);
}

__global__ void advance_kernel(const mel_dev* devs, int nsamp)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s < nsamp) devs[s].time2[0] = devs[s].time2[0] + devs[s].dt[0];
}

// ------------------------------------------------------------------------------------------
// monitor: kinetic energy (Monitoring.h:528-531), mass-weighted mean displacement (88-101),
// active contact elements; block partials then a fixed-order final sum (deterministic)
// ------------------------------------------------------------------------------------------
#define MON_BLOCKS 148
__global__ void monitor_partial_kernel(mel_dev d, double* part)
{
    __shared__ double s[5][256];
    double ke = 0., ux = 0., uy = 0., mt = 0., act = 0.;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < d.nn; i += gridDim.x * blockDim.x) {
        double2 v = d.v[i], m = d.mass[i], u = d.u[i];
        ke += 0.5 * v.x * v.x * m.x + 0.5 * v.y * v.y * m.y;
        ux += u.x * m.x; uy += u.y * m.y; mt += m.x;      // rigid nodes carry zero mass
    }
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < d.ncont; c += gridDim.x * blockDim.x)
        if (d.cont[c].fx != 0. || d.cont[c].fy != 0.) act += 1.;
    s[0][threadIdx.x] = ke; s[1][threadIdx.x] = ux; s[2][threadIdx.x] = uy; s[3][threadIdx.x] = mt; s[4][threadIdx.x] = act;
    __syncthreads();
    for (int w = 128; w > 0; w >>= 1) {
        if (threadIdx.x < w)
            for (int k = 0; k < 5; k++) s[k][threadIdx.x] += s[k][threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x < 5) part[threadIdx.x * MON_BLOCKS + blockIdx.x] = s[threadIdx.x][0];
}

__global__ void monitor_final_kernel(mel_dev d, const double* part, const int* rigid_ids, int nrigid, double* out)
{
    if (threadIdx.x == 0) {
        double t[5] = { 0., 0., 0., 0., 0. };
        for (int k = 0; k < 5; k++)
            for (int b = 0; b < MON_BLOCKS; b++) t[k] += part[k * MON_BLOCKS + b];
        out[0] = t[0];
        out[1] = t[3] > 0 ? t[1] / t[3] : 0.;
        out[2] = t[3] > 0 ? t[2] / t[3] : 0.;
        out[3] = t[4];
        for (int r = 0; r < nrigid && r < 4; r++) {
            const double* rf = d.rf + 15 * rigid_ids[r];
            out[4 + 4 * r] = rf[0]; out[5 + 4 * r] = rf[1]; out[6 + 4 * r] = rf[6]; out[7 + 4 * r] = rf[7];
        }
    }
}

// ------------------------------------------------------------------------------------------
// Update_contact_pressures (Code/Proximity.h:1014-1069): every contact adds f / length to its
// slave border entry and subtracts f / length * shapeM1 (shapeM2) from the master entries at the
// ends of its segment.  The reference adds them in list order, contact by contact (slave, then
// the two master entries), so each border entry gathers its contributions, sorts them by
// (contact, role) and adds them in that order.
// ------------------------------------------------------------------------------------------
__device__ __forceinline__ void pressure_push(const mel_dev& d, int e, int v)
{
    if (e < 0 || e >= d.ne) { set_err(d, MEL_E_BOUNDS); return; }
    const int slot = atomicAdd(&d.cp_cnt[e], 1);
    if (slot < MEL_PRESSURE_CAP) d.cp_item[(size_t)e * MEL_PRESSURE_CAP + slot] = v;
    else set_err(d, MEL_E_PRESSURE);
}

__global__ void pressure_clear_kernel(mel_dev d)
{
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e < d.ne) d.cp_cnt[e] = 0;
}

__global__ void pressure_push_kernel(mel_dev d)
{
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= d.ncont) return;
    const mel_contact& k = d.cont[c];
    if (k.bodyS < 0 || k.bodyS >= d.nb || k.bodyM < 0 || k.bodyM >= d.nb) { set_err(d, MEL_E_BOUNDS); return; }
    const int eS = d.bd_e0[d.b_bd0[k.bodyS] + k.borderS] + k.border_nodeS;
    const int eM = d.bd_e0[d.b_bd0[k.bodyM] + k.borderM] + k.segmentM;
    pressure_push(d, eS, c << 2);
    pressure_push(d, eM, (c << 2) | 1);
    pressure_push(d, eM + 1, (c << 2) | 2);
}

__global__ void pressure_sum_kernel(mel_dev d)
{
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= d.ne) return;
    const int n = min(d.cp_cnt[e], MEL_PRESSURE_CAP);
    int v[MEL_PRESSURE_CAP];
    for (int i = 0; i < n; i++) {                         // insertion sort: a handful of items
        const int x = d.cp_item[(size_t)e * MEL_PRESSURE_CAP + i];
        int j = i;
        while (j > 0 && v[j - 1] > x) { v[j] = v[j - 1]; j--; }
        v[j] = x;
    }
    double px = 0., py = 0.;
    for (int i = 0; i < n; i++) {
        const mel_contact& k = d.cont[v[i] >> 2];
        const int role = v[i] & 3;
        const double il = 1. / k.length;
        if (role == 0) { px += k.fx * il; py += k.fy * il; }
        else {
            const double sh = k.shapeM[role];
            px -= k.fx * il * sh;
            py -= k.fy * il * sh;
        }
    }
    d.cpx[e] = px;
    d.cpy[e] = py;
}

} // namespace mel

void mel_launch_contact_pressures(const mel_dev& d, cudaStream_t s)
{
    if (d.ne <= 0) return;
    mel::pressure_clear_kernel<<<(d.ne + 255) / 256, 256, 0, s>>>(d);
    if (d.ncont > 0) mel::pressure_push_kernel<<<(d.ncont + 127) / 128, 128, 0, s>>>(d);
    mel::pressure_sum_kernel<<<(d.ne + 127) / 128, 128, 0, s>>>(d);
}

namespace mel {
// Body::Update_damping_forces (Code/Body.h:1057-1154): each degree of freedom subtracts its terms
// v_param(source) * c in matrix-entry order, the order the reference's loop over the entries adds
// them in; one thread per degree of freedom
__global__ void __launch_bounds__(256) damping_kernel(mel_dev d)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= 2 * d.nn) return;
    const int a = d.dmp_ptr[k], e = d.dmp_ptr[k + 1];
    if (a == e) return;
    const double* vp = reinterpret_cast<const double*>(d.vp);
    double f = 0.;
    for (int j = a; j < e; j++) f = f - vp[d.dmp_src[j]] * d.dmp_c[j];
    reinterpret_cast<double*>(d.fdamp)[k] = f;
}
}  // namespace mel

namespace mel {
// Body::Update_alid_forces (Code/Body.h:1163-1296), one CTA per body with a layer: the reference
// velocity of each direction from its history (the first interval holding T; 0 when none does,
// where the reference reads past its vector), then per degree of freedom the nodal term
// -beta m (v - pv) followed by its stiffness terms -(v_param(source) - pv(source)) d in the
// order the reference's entry loop adds them; a direction without history keeps a zero force
__global__ void __launch_bounds__(256) alid_kernel(mel_dev d, int parity, double T, int use_T)
{
    const int b = d.alid_b[blockIdx.x];
    __shared__ double s_pv[2];
    __shared__ int s_fl[2];
    if (threadIdx.x < 2) {
        const int dir = threadIdx.x;
        const double t = use_T ? T : d.time2[parity];
        const int h0 = d.alid_hptr[2 * b + dir], h1 = d.alid_hptr[2 * b + dir + 1];
        double pv = 0.;
        for (int k = h0; k + 1 < h1; k++) {
            const double t0 = d.alid_ht[k], p0 = d.alid_hv[k], t1 = d.alid_ht[k + 1], p1 = d.alid_hv[k + 1];
            if ((t0 <= t) & (t <= t1)) { pv = p0 + (p1 - p0) / (t1 - t0) * (t - t0); break; }
        }
        s_pv[dir] = pv;
        s_fl[dir] = h1 > h0;
    }
    __syncthreads();
    const double* v = reinterpret_cast<const double*>(d.v);
    const double* vp = reinterpret_cast<const double*>(d.vp);
    const double* m = reinterpret_cast<const double*>(d.mass);
    double* f = reinterpret_cast<double*>(d.falid);
    for (int k = 2 * d.b_node0[b] + threadIdx.x; k < 2 * d.b_node0[b + 1]; k += blockDim.x) {
        const int dir = k & 1;
        double a = s_fl[dir] ? -d.alid_beta[k >> 1] * m[k] * (v[k] - s_pv[dir]) : 0.;
        for (int j = d.al_ptr[k]; j < d.al_ptr[k + 1]; j++) {
            const int src = d.al_src[j];
            a += -(vp[src] - s_pv[src & 1]) * d.al_c[j];
        }
        f[k] = a;
    }
}
}  // namespace mel

void mel_launch_alid(const mel_dev& d, int parity, double T, int use_T, cudaStream_t s)
{
    if (!d.falid || d.n_alid == 0) return;
    mel::alid_kernel<<<d.n_alid, 256, 0, s>>>(d, parity, T, use_T);
}

void mel_launch_damping(const mel_dev& d, cudaStream_t s)
{
    if (!d.fdamp || d.nn == 0) return;
    mel::damping_kernel<<<(2 * d.nn + 255) / 256, 256, 0, s>>>(d);
}

void mel_launch_contact(const mel_dev& d, double law_dt_scale, cudaStream_t s)
{
    int total = d.ncont + d.ne;
    if (total <= 0) return;
    mel::contact_kernel<<<(total + 127) / 128, 128, 0, s>>>(d, law_dt_scale, 0);
}

void mel_launch_czm_init(const mel_dev& d, cudaStream_t s)
{
    if (d.ncont <= 0) return;
    mel::contact_kernel<<<(d.ncont + 127) / 128, 128, 0, s>>>(d, 1.0, 1);
}

size_t mel_body_smem_bytes(int max_nodes, int max_image_bytes, int mixed, int stages)
{
    size_t base = 3 * sizeof(double2) * (size_t)max_nodes + MEL_BAR_BYTES;
    if (mixed) base += sizeof(float2) * (size_t)((max_nodes + 1) & ~1);
    size_t stage = (size_t)stages * (size_t)max_image_bytes;
    size_t post = (5 * sizeof(double2) + 6 * sizeof(double)) * (size_t)max_nodes;
    size_t rigid = (64 + 6 * MEL_RIGID_BATCH) * sizeof(double);
    size_t r = base + (stage > post ? stage : post);
    return r > rigid ? r : rigid;
}

void mel_launch_batch_step(const mel_dev* devs, const int* thr0, int nthr, const int* cta0, int ncta_small, int ncta,
                           int nsamp, int mixed, size_t smem_small, size_t smem, cudaStream_t s)
{
    if (nthr > 0) mel::contact_kernel_batch<<<(nthr + 127) / 128, 128, 0, s>>>(devs, thr0, nsamp, 1.0);
    // members whose bodies fit two CTAs per SM first, in their own launch, then the others
    if (ncta_small > 0) {
        if (mixed) mel::body_kernel_batch<true><<<ncta_small, MEL_BODY_THREADS, smem_small, s>>>(devs, cta0, nsamp, 0);
        else mel::body_kernel_batch<false><<<ncta_small, MEL_BODY_THREADS, smem_small, s>>>(devs, cta0, nsamp, 0);
    }
    if (ncta > ncta_small) {
        if (mixed) mel::body_kernel_batch<true><<<ncta - ncta_small, MEL_BODY_THREADS, smem, s>>>(devs, cta0, nsamp, ncta_small);
        else mel::body_kernel_batch<false><<<ncta - ncta_small, MEL_BODY_THREADS, smem, s>>>(devs, cta0, nsamp, ncta_small);
    }
    mel::advance_kernel<<<(nsamp + 127) / 128, 128, 0, s>>>(devs, nsamp);
}

void mel_launch_body(const mel_dev& d, int parity, int nblocks, size_t smem, cudaStream_t s, int nwide)
{
    if (nblocks > 0) {
        if (d.precision == MEL_PREC_MIXED) mel::body_kernel<true><<<nblocks, MEL_BODY_THREADS, smem, s>>>(d, parity);
        else mel::body_kernel<false><<<nblocks, MEL_BODY_THREADS, smem, s>>>(d, parity);
    }
    if (nwide > 0) {
        const int set_time = nblocks > 0 ? 0 : 1;
        if (d.precision == MEL_PREC_MIXED) mel::body_kernel_wide<true><<<nwide, MEL_BODY_THREADS, smem, s>>>(d, parity, nblocks, set_time);
        else mel::body_kernel_wide<false><<<nwide, MEL_BODY_THREADS, smem, s>>>(d, parity, nblocks, set_time);
    }
}

void mel_launch_body_adaptive(const mel_dev& d, double T0, double Tf, int nblocks, size_t smem, cudaStream_t s, int nwide)
{
    if (nblocks > 0) {
        if (d.precision == MEL_PREC_MIXED) mel::body_kernel_adaptive<true><<<nblocks, MEL_BODY_THREADS, smem, s>>>(d, T0, Tf);
        else mel::body_kernel_adaptive<false><<<nblocks, MEL_BODY_THREADS, smem, s>>>(d, T0, Tf);
    }
    if (nwide > 0) {
        if (d.precision == MEL_PREC_MIXED) mel::body_kernel_adaptive_wide<true><<<nwide, MEL_BODY_THREADS, smem, s>>>(d, T0, Tf, nblocks);
        else mel::body_kernel_adaptive_wide<false><<<nwide, MEL_BODY_THREADS, smem, s>>>(d, T0, Tf, nblocks);
    }
}

void mel_launch_error_reduce(const mel_dev& d, double* out, cudaStream_t s)
{
    mel::error_reduce_kernel<<<1, 32, 0, s>>>(d, out);
}

namespace mel {
// Body::Restore of a rigid body's own kinematics (Code/Body.h:2650-2658): current position,
// displacement and velocity; its accelerations, driven values and mass-scaling factor are not
// part of the snapshot
__global__ void rigid_restore_kernel(mel_dev d, const double* rg_snap)
{
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= d.nb || d.b_type[b] != MEL_BODY_RIGID) return;
    const double* s = rg_snap + MEL_RIGID_NF * (size_t)b;
    double* r = d.rg + MEL_RIGID_NF * (size_t)b;
    const int f[9] = { MEL_RG_XC, MEL_RG_YC, MEL_RG_RC, MEL_RG_XD, MEL_RG_YD, MEL_RG_RD, MEL_RG_XV, MEL_RG_YV, MEL_RG_RV };
    for (int k = 0; k < 9; k++) r[f[k]] = s[f[k]];
}
}  // namespace mel

namespace mel {
// Update_bc(Time) of every body's driven borders (the set-up call of Code/main.cpp:104-127)
__global__ void drivendof_kernel(mel_dev d, double T)
{
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b < d.nb) body_drivendof(d, b, T, d.drv + 8 * (size_t)b);
}
}  // namespace mel

void mel_launch_drivendof(const mel_dev& d, double T, cudaStream_t s)
{
    mel::drivendof_kernel<<<(d.nb + 127) / 128, 128, 0, s>>>(d, T);
}

void mel_launch_rigid_restore(const mel_dev& d, const double* rg_snap, cudaStream_t s)
{
    mel::rigid_restore_kernel<<<(d.nb + 127) / 128, 128, 0, s>>>(d, rg_snap);
}

void mel_launch_monitor(const mel_dev& d, double* part, const int* rigid_ids, int nrigid, double* out, cudaStream_t s)
{
    mel::monitor_partial_kernel<<<MON_BLOCKS, 256, 0, s>>>(d, part);
    mel::monitor_final_kernel<<<1, 32, 0, s>>>(d, part, rigid_ids, nrigid, out);
}

// The attribute is per kernel and device, shared by every handle of the process: it is only ever
// raised (to the largest size any handle needs), never lowered under another handle's launches.
int mel_body_kernel_configure(size_t smem)
{
    static std::mutex mu;
    static size_t configured[64] = {};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return MEL_ERR_CUDA;
    std::lock_guard<std::mutex> lock(mu);
    if (smem <= configured[dev]) return MEL_OK;
    if (cudaFuncSetAttribute(mel::body_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess ||
        cudaFuncSetAttribute(mel::body_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess ||
        cudaFuncSetAttribute(mel::body_kernel_batch<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess ||
        cudaFuncSetAttribute(mel::body_kernel_batch<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess ||
        cudaFuncSetAttribute(mel::body_kernel_adaptive<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess ||
        cudaFuncSetAttribute(mel::body_kernel_adaptive<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess ||
        cudaFuncSetAttribute(mel::body_kernel_wide<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess ||
        cudaFuncSetAttribute(mel::body_kernel_wide<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess ||
        cudaFuncSetAttribute(mel::body_kernel_adaptive_wide<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess ||
        cudaFuncSetAttribute(mel::body_kernel_adaptive_wide<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess) {
        mel_set_cuda_error(cudaGetLastError(), "cudaFuncSetAttribute(body_kernel)", __FILE__, __LINE__);
        return MEL_ERR_CUDA;
    }
    configured[dev] = smem;
    return MEL_OK;
}
