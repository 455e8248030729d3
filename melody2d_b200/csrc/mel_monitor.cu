// Monitoring (Code/Monitoring.h:8-559) on the device: after every accepted step the solver's stream
// runs mon_body_kernel (one warp per body: the body's sums that the whole-sample quantities add up)
// and mon_row_kernel (one thread: the monitored entries in list order, then the energy and boundary
// blocks), which appends the row to a device buffer that the host drains at save time
// (Write_monitoring, Code/IO.h:2644-2668).  No host download happens per step.
//
// Exactness: every quantity of one node, one body or one border is computed in the reference's
// operation order (a single thread walks the body's nodes in index order), so it equals the
// reference's value bit for bit on the same state.  The three sums over the whole sample (kinetic
// energy of MONITOR_ENERGY, Dwork, and Energy Kinetic of all bodies) add per-body partial sums,
// which changes the association of the reference's single running sum: they agree with it to a
// few units in the last place, far inside the 10 significant digits MONITORING.asc keeps.
#include "mel_internal.h"

namespace mel {

// per body b: part[3b] = sum over its nodes of 1/2 m v^2 with the nodal velocities (the terms of
// Monitoring.h:528-531), part[3b+1] = the body's Energy Kinetic term (Monitoring.h:398-412:
// velocity parameters of a deformable body's nodes, or the rigid body's translation and rotation),
// part[3b+2] = the body's Dwork terms (Monitoring.h:516-526) with Deltat = dt
__global__ void __launch_bounds__(256) mon_body_kernel(mel_dev d, double dt, double* part)
{
    const int b = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    const int lane = threadIdx.x & 31;
    if (b >= d.nb) return;
    const int n0 = d.b_node0[b], n1 = d.b_node0[b + 1];
    const bool def = d.b_type[b] == MEL_BODY_DEFORMABLE;
    double ke = 0., kp = 0., dw = 0.;
    for (int i = n0 + lane; i < n1; i += 32) {
        const double2 v = d.v[i], m = d.mass[i];
        ke += 0.5 * v.x * v.x * m.x;
        ke += 0.5 * v.y * v.y * m.y;
        if (def) {
            const double2 w = d.vp[i];
            kp += 0.5 * w.x * w.x * m.x;
            kp += 0.5 * w.y * w.y * m.y;
        }
    }
    const int e0 = d.bd_e0[d.b_bd0[b]], e1 = d.bd_e0[d.b_bd0[b + 1]];
    for (int e = e0 + lane; e < e1; e += 32) {
        const double2 p = d.e_bcp[e], v = d.v[n0 + d.e_node[e]];
        dw += (p.x * v.x + p.y * v.y) * d.e_len[e] * dt;
    }
    for (int o = 16; o; o >>= 1) {
        ke += __shfl_xor_sync(0xffffffffu, ke, o);
        kp += __shfl_xor_sync(0xffffffffu, kp, o);
        dw += __shfl_xor_sync(0xffffffffu, dw, o);
    }
    if (lane == 0) {
        if (!def) {
            const double* rg = d.rg + (size_t)MEL_RIGID_NF * b;
            kp = 0.;
            kp += 0.5 * rg[MEL_RG_XV] * rg[MEL_RG_XV] * rg[MEL_RG_MASS];
            kp += 0.5 * rg[MEL_RG_YV] * rg[MEL_RG_YV] * rg[MEL_RG_MASS];
            kp += 0.5 * rg[MEL_RG_RV] * rg[MEL_RG_RV] * rg[MEL_RG_INERTIA];
        }
        part[3 * b] = ke;
        part[3 * b + 1] = kp;
        part[3 * b + 2] = dw;
    }
}

// nodal force of kind s (Read_spy_line's force index: total, internal, contact, body, Dirichlet,
// Neumann, damping, ALID) of global node i of body b, as Node stores it after Sum_up_forces
// (Code/Body.h:1974-2012 copies a rigid body's forces to its nodes)
__device__ double2 node_force(const mel_dev& d, int b, int i, int s)
{
    const bool rigid = d.b_type[b] == MEL_BODY_RIGID;
    const double* rf = d.rf + 15 * b;
    switch (s) {
    case 0: return d.o_ftot[i];
    case 1: return d.o_fint[i];
    case 2: return d.o_fcon[i];
    case 3: {
        if (rigid) return make_double2(rf[3], rf[4]);
        const bool ng = d.b_status[b] == MEL_STATUS_NOGRAVITY;
        const double2 m = d.mass[i];
        return make_double2(m.x * (ng ? 0. : d.gx), m.y * (ng ? 0. : d.gy));   // Code/Body.h:916-922
    }
    case 4: return d.o_fdir[i];
    case 5: return d.o_fneu[i];
    case 6: return rigid ? make_double2(rf[12], rf[13]) : (d.fdamp ? d.fdamp[i] : make_double2(0., 0.));
    case 7: return rigid ? make_double2(0., 0.) : (d.falid ? d.falid[i] : make_double2(0., 0.));
    default: return make_double2(0., 0.);
    }
}

// Body::Update_damage (Code/Body.h:2667-2700) of body b: per border node the smallest internal[0]
// of the body's contact elements on that node that carry internal variables (1 when none does),
// averaged over the border nodes in border order, never below the body's previous value, which it
// replaces (d.b_damage); one thread
__device__ double body_damage(const mel_dev& d, int b)
{
    double total_nodes = 0., dmg = 0.;
    const double previous = d.b_damage[b];
    const int c0 = d.b_cont0[b], c1 = d.b_cont0[b + 1];
    for (int g = d.b_bd0[b]; g < d.b_bd0[b + 1]; g++) {
        const int i = g - d.b_bd0[b];
        const int nbn = d.bd_e0[g + 1] - d.bd_e0[g];
        total_nodes += nbn;
        for (int j = 0; j < nbn; j++) {
            double v = 1.;
            for (int k = c0; k < c1; k++) {
                const mel_contact& c = d.cont[k];
                if (c.borderS == i && c.border_nodeS == j && c.nb_internal > 0 && c.internal[0] < v) v = c.internal[0];
            }
            dmg += v;
        }
    }
    dmg = dmg / total_nodes;
    if (dmg < previous) dmg = previous;
    d.b_damage[b] = dmg;
    return dmg;
}

// one row of Monitoring (Code/Monitoring.h:8-559) into row[1..], its length into row[0]
__global__ void mon_row_kernel(mel_dev d, const mel_mon_op* ops, int nops, int energy, int boundaries,
                               const double* part, double* row, mel_mon_head hd)
{
    if (threadIdx.x != 0) return;
    int c = 1;
    row[c++] = hd.iteration; row[c++] = hd.time; row[c++] = hd.dt;
    row[c++] = hd.neval; row[c++] = hd.max_error; row[c++] = hd.mean_error;
    // x, y, r and m live across entries as in the reference, where an entry that does not assign
    // one of them reads the value the previous entry left (never-assigned values start at 0)
    double x = 0., y = 0., r = 0., m = 0.;
    for (int k = 0; k < nops; k++) {
        const mel_mon_op o = ops[k];
        if (o.type <= 3) {
            // Position, Displacement, Velocity, Acceleration (Monitoring.h:33-192)
            const double2* a = o.type == 0 ? d.x : o.type == 1 ? d.u : o.type == 2 ? d.v : d.a;
            const int rx = o.type == 0 ? MEL_RG_XC : o.type == 1 ? MEL_RG_XD : o.type == 2 ? MEL_RG_XV : MEL_RG_XA;
            const int n0 = d.b_node0[o.body];
            if (o.node >= 0) {
                const double2 p = a[n0 + o.node];
                x = p.x; y = p.y;
            } else if (d.b_type[o.body] == MEL_BODY_DEFORMABLE) {
                x = 0.; y = 0.; m = 0.;
                for (int j = n0; j < d.b_node0[o.body + 1]; j++) {
                    const double2 p = a[j], w = d.mass[j];
                    x += p.x * w.x;
                    y += p.y * w.y;
                    m += w.x;
                }
                x /= m;
                y /= m;
            } else {
                const double* rg = d.rg + (size_t)MEL_RIGID_NF * o.body;
                x = rg[rx]; y = rg[rx + 1]; r = rg[rx + 2];
            }
            if (o.kind == 0) row[c++] = x;
            else if (o.kind == 1) row[c++] = y;
            else if (o.type == 0) { if (o.kind == 2) row[c++] = r; }
            else if (o.kind == 2) row[c++] = sqrt(x * x + y * y);   // pow(.,0.5): both correctly rounded
            else if (o.kind == 3) row[c++] = r;
        } else if (o.type == 4) {
            // Force (Monitoring.h:193-338): o.sub = force kind, o.body, o.node
            const int b = o.body;
            if (o.node >= 0) {
                const double2 f = node_force(d, b, d.b_node0[b] + o.node, o.sub);
                x = f.x; y = f.y;
            } else if (d.b_type[b] == MEL_BODY_DEFORMABLE) {
                // the reference bounds this loop by the node count of body number o.sub
                // (Monitoring.h:232); the host checked that it stays inside body b
                x = 0.; y = 0.;
                const int n0 = d.b_node0[b], cnt = d.b_node0[o.sub + 1] - d.b_node0[o.sub];
                for (int j = 0; j < cnt; j++) {
                    const double2 f = node_force(d, b, n0 + j, o.sub);
                    x += f.x;
                    y += f.y;
                }
            } else {
                const double* rf = d.rf + 15 * b;
                const int s = o.sub;
                if (s == 0) { x = d.rtot[3 * b]; y = d.rtot[3 * b + 1]; r = d.rtot[3 * b + 2]; }
                else if (s >= 2 && s <= 6) { const int q = 3 * (s - 2); x = rf[q]; y = rf[q + 1]; r = rf[q + 2]; }
            }
            if (o.kind == 0) row[c++] = x;
            else if (o.kind == 1) row[c++] = y;
            else if (o.kind == 2) row[c++] = sqrt(x * x + y * y);
            else if (o.kind == 3) row[c++] = r;
        } else if (o.type == 7) {
            // Contact (Monitoring.h:362-382): the body's first contact element of that slave node
            for (int j = d.b_cont0[o.body]; j < d.b_cont0[o.body + 1]; j++) {
                const mel_contact& e = d.cont[j];
                if (e.borderS == o.border && e.border_nodeS == o.bnode) {
                    if (o.kind == 0) row[c++] = e.gapn;
                    else if (o.kind == 1) row[c++] = e.gapt;
                    else if (o.kind == 2) row[c++] = e.xsi;
                    else if (o.kind == 3) row[c++] = e.xnorm;
                    else if (o.kind == 4) row[c++] = e.ynorm;
                    else if (o.kind == 5) row[c++] = e.internal[0];
                    break;
                }
            }
        } else if (o.type == 8) {
            // Damage (Monitoring.h:385-390): Update_damage of the body, then its damage
            row[c++] = body_damage(d, o.body);
        } else if (o.type == 9) {
            // Energy (Monitoring.h:390-458); the elastic energy of both material laws is zero
            // (Code/Model.h:19-73 set energy = 0), so Deformation entries read +0
            x = 0.;
            if (o.body >= 0) {
                if (o.kind == 0) {
                    if (d.b_type[o.body] == MEL_BODY_DEFORMABLE) {
                        for (int j = d.b_node0[o.body]; j < d.b_node0[o.body + 1]; j++) {
                            const double2 w = d.vp[j], ms = d.mass[j];
                            x += 0.5 * w.x * w.x * ms.x;
                            x += 0.5 * w.y * w.y * ms.y;
                        }
                    } else {
                        x = part[3 * o.body + 1];
                    }
                }
            } else if (o.body == -1 && o.kind == 0) {
                for (int b = 0; b < d.nb; b++) x += part[3 * b + 1];
            }
            row[c++] = x;
        } else if (o.type == 10) {
            // Work (Monitoring.h:459-503)
            if (o.body >= 0) {
                if (o.kind >= 0 && o.kind < 7) row[c++] = d.works[7 * o.body + o.kind];
            } else if (o.body == -1) {
                x = 0.;
                if (o.kind >= 0 && o.kind < 7)
                    for (int b = 0; b < d.nb; b++) x += d.works[7 * b + o.kind];
                row[c++] = x;
            }
        }
        // other entry types add no column (Monitoring.h handles types 0-10 only)
    }
    if (energy) {
        // MONITOR_ENERGY (Monitoring.h:508-537): Dwork, elastic energy (zero), kinetic energy
        double dw = 0., ke = 0.;
        for (int b = 0; b < d.nb; b++) { dw += part[3 * b + 2]; ke += part[3 * b]; }
        row[c++] = dw;
        row[c++] = 0.;
        row[c++] = ke;
    }
    if (boundaries) {
        // MONITOR_BOUNDARIES (Monitoring.h:539-556): border 0 of body 0 and border 1 of body 1;
        // the reference leaves the four sums uninitialised, they start at 0 here
        double f[4] = { 0., 0., 0., 0. };
        for (int s = 0; s < 2; s++) {
            const int g = d.b_bd0[s] + s;
            for (int e = d.bd_e0[g]; e < d.bd_e0[g + 1]; e++) {
                const double2 p = d.e_bcp[e];
                f[2 * s] += p.x * d.e_len[e];
                f[2 * s + 1] += p.y * d.e_len[e];
            }
        }
        for (int k = 0; k < 4; k++) row[c++] = f[k];
    }
    row[0] = (double)(c - 1);
}

// Update_status (Code/Proximity.h:550-1007), one thread, entries in order.  e = the entry (type,
// then the fields Read_spy_line stores, the comparison 0 below / 1 equal / 2 above, the threshold).
// x, y, r carry over between entries of one call as in the reference (they start at 0 each call).
// sets a body inactive.  The reference stops clearing the send list of an inactive body but goes
// on sending it (Code/Solver.h:37-61: Initialize_contact_forces skipped, Send_contact_forces not),
// so a body switched off while one of its contact elements carries a force keeps pushing that force
// onto its masters for the rest of the run; that is reported rather than reproduced
__device__ void deactivate(const mel_dev& d, int body)
{
    if (d.b_status[body] != MEL_STATUS_INACTIVE) {
        for (int j = d.b_cont0[body]; j < d.b_cont0[body + 1]; j++)
            if (d.cont[j].bodyM != body && (d.cont[j].fx != 0. || d.cont[j].fy != 0.)) {
                atomicCAS(d.err + MEL_E_DEACT, 0u, (unsigned)body + 1u);
                break;
            }
    }
    d.b_status[body] = MEL_STATUS_INACTIVE;
}

__global__ void status_kernel(mel_dev d, const double* entries, int n)
{
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    double x = 0., y = 0., r = 0., m = 0.;
    for (int k = 0; k < n; k++) {
        const double* e = entries + MEL_DEACT_NF * k;
        const int type = (int)e[0], kind = (int)e[1];
        int body, mode;
        double thr;
        if (type <= 3) {
            // Position, Displacement, Velocity, Acceleration of a node or a whole body
            body = (int)e[2];
            const int node = (int)e[3];
            mode = (int)e[4]; thr = e[5];
            const double2* a = type == 0 ? d.x : type == 1 ? d.u : type == 2 ? d.v : d.a;
            const int rx = type == 0 ? MEL_RG_XC : type == 1 ? MEL_RG_XD : type == 2 ? MEL_RG_XV : MEL_RG_XA;
            const int n0 = d.b_node0[body];
            if (node >= 0) {
                const double2 p = a[n0 + node];
                x = p.x; y = p.y;
            } else if (d.b_type[body] == MEL_BODY_DEFORMABLE) {
                x = 0.; y = 0.; m = 0.;
                for (int j = n0; j < d.b_node0[body + 1]; j++) {
                    const double2 p = a[j], w = d.mass[j];
                    x += p.x * w.x;
                    y += p.y * w.y;
                    m += w.x;
                }
                x /= m;
                y /= m;
            } else {
                const double* rg = d.rg + (size_t)MEL_RIGID_NF * body;
                x = rg[rx]; y = rg[rx + 1]; r = rg[rx + 2];
            }
        } else if (type == 4) {
            // Force: e[2] = force kind, e[3] = body, e[4] = node
            const int fk = (int)e[2];
            body = (int)e[3];
            const int node = (int)e[4];
            mode = (int)e[5]; thr = e[6];
            if (node >= 0) {
                if (fk <= 6) {
                    const double2 f = node_force(d, body, d.b_node0[body] + node, fk);
                    x = f.x; y = f.y;
                }
            } else if (d.b_type[fk] == MEL_BODY_DEFORMABLE) {
                // the reference tests the type of body number <force kind>, walks as many nodes as
                // that body has, and adds total forces (kind 0) or damping forces (kind 1) of body
                // e[3] (Code/Proximity.h:866-882); the host checked that the walk stays inside it
                x = 0.; y = 0.;
                const int n0 = d.b_node0[body], cnt = d.b_node0[fk + 1] - d.b_node0[fk];
                for (int j = 0; j < cnt; j++) {
                    if (fk == 0) { const double2 f = node_force(d, body, n0 + j, 0); x += f.x; y += f.y; }
                    else if (fk == 1) { const double2 f = node_force(d, body, n0 + j, 6); x += f.x; y += f.y; }
                }
            } else {
                const double* rf = d.rf + 15 * body;
                if (fk == 0) { x = d.rtot[3 * body]; y = d.rtot[3 * body + 1]; r = d.rtot[3 * body + 2]; }
                else if (fk >= 2 && fk <= 6) { const int q = 3 * (fk - 2); x = rf[q]; y = rf[q + 1]; r = rf[q + 2]; }
            }
        } else if (type == 8) {
            // Damage (Code/Proximity.h:988-998): e = {8, body, mode, threshold}
            body = (int)e[1];
            mode = (int)e[2]; thr = e[3];
            const double dm = body_damage(d, body);
            if ((mode == 0 && dm <= thr) || (mode == 1 && dm == thr) || (mode == 2 && dm >= thr)) deactivate(d, body);
            continue;
        } else {
            continue;
        }
        double v;
        if (kind == 0) v = x;
        else if (kind == 1) v = y;
        else if (kind == 2) v = type == 0 ? r : sqrt(x * x + y * y);    // pow(.,0.5): both correctly rounded
        else if (kind == 3 && type != 0) v = r;
        else continue;                                                 // no comparison in the reference
        if ((mode == 0 && v <= thr) || (mode == 1 && v == thr) || (mode == 2 && v >= thr)) deactivate(d, body);
    }
}

}  // namespace mel

void mel_launch_status(const mel_dev& d, const double* entries, int n, cudaStream_t s)
{
    if (n > 0) mel::status_kernel<<<1, 32, 0, s>>>(d, entries, n);
}

void mel_launch_monitor(const mel_dev& d, const mel_mon_op* ops, int nops, int energy, int boundaries,
                        double* part, double* row, const mel_mon_head& hd, cudaStream_t s)
{
    if (d.nb > 0) mel::mon_body_kernel<<<(d.nb + 7) / 8, 256, 0, s>>>(d, hd.dt, part);
    mel::mon_row_kernel<<<1, 32, 0, s>>>(d, ops, nops, energy, boundaries, part, row, hd);
}
