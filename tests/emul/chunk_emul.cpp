// CPU model of the body kernel's Gauss-point pass over the chunk images (test infrastructure).
// It reads each image exactly as the kernel does (header, sections, slot records, row tables,
// pull records), checks every index it follows against the image and body bounds, and returns
// the internal nodal forces, so a test can compare them with the oracle bit for bit.
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <utility>
#include <vector>
#include "mel_chunks.h"

static char g_err[512];
void mel_set_error(const char* fmt, ...)
{
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof g_err, fmt, ap);
    va_end(ap);
}

extern "C" const char* emul_error() { return g_err; }

// up: 2 doubles per node (displacements the pass reads); f: 2 doubles per node (output, rigid
// nodes left at zero); stats: [chunks, stored entries, padding entries, largest image bytes].
// Returns 0, or a positive code when an index read from an image is out of bounds.
extern "C" int emul_internal_forces(const mel_model_desc* d, int ecap, const double* up, double* f, long long* stats)
{
    mel_chunk_set CS;
    if (mel_build_chunks(d, ecap, CS) != MEL_OK) return 100;
    stats[0] = (long long)CS.chunks.size(); stats[1] = CS.n_entries; stats[2] = CS.n_pad; stats[3] = CS.img_max;
    memset(f, 0, sizeof(double) * 2 * (size_t)d->n_nodes);
    for (int b = 0; b < d->n_bodies; b++) {
        if (d->body_type[b] != MEL_BODY_DEFORMABLE) continue;
        const int n0 = d->body_node_ptr[b], n = d->body_node_ptr[b + 1] - n0;
        const int mat = d->body_material[b];
        const int mtype = d->material_type[mat];
        const double Mu = d->material_params[MEL_MAT_NPARAM * mat + 3];
        const double Lam = d->material_params[MEL_MAT_NPARAM * mat + 4];
        std::vector<double> sf(2 * (size_t)n, 0.);
        std::vector<uint8_t> buf;
        for (int ci = CS.b_chunk0[b]; ci < CS.b_chunk0[b + 1]; ci++) {
            const mel_chunk& c = CS.chunks[ci];
            if (c.bytes % 16 || c.img % 16 || c.bytes > CS.img_max) return 1;
            buf.assign(CS.img.begin() + c.img, CS.img.begin() + c.img + c.bytes);
            int hdr[4];
            memcpy(hdr, buf.data(), sizeof hdr);
            if (hdr[0] > MEL_CHUNK_GP_FP64 || hdr[1] % 8 || hdr[1] > ecap || hdr[3] > 1024) return 2;
            const int wide = n > MEL_MAX_BODY_NODES ? 1 : 0;
            const mel_chunk_layout L = mel_chunk_sections(hdr[0], hdr[1], hdr[2], hdr[3], 16, wide);
            if (L.bytes != c.bytes) return 3;
            double* sp = reinterpret_cast<double*>(buf.data() + L.dN);
            const uint16_t* sidx = reinterpret_cast<const uint16_t*>(buf.data() + L.idx);
            const uint16_t* stpos = reinterpret_cast<const uint16_t*>(buf.data() + L.tpos);
            const double* sc0 = reinterpret_cast<const double*>(buf.data() + L.c0);
            const uint32_t* sgpm = reinterpret_cast<const uint32_t*>(buf.data() + L.gpm);
            const uint32_t* stn = reinterpret_cast<const uint32_t*>(buf.data() + L.tn);
            const uint16_t* sroff = reinterpret_cast<const uint16_t*>(buf.data() + L.roff);
            const int ne = hdr[1];
            for (int t = 0; t < hdr[0]; t++) {
                const uint32_t gm = sgpm[t];
                const int r0 = (int)(gm & 0x3ffu), lane = (int)((gm >> 10) & 0x1fu), ns = (int)(gm >> 15);
                if (r0 + ns > hdr[3] || lane != t % 32) return 4;
                // the kernel computes every position from the group's first entry, its width m and
                // the row's lane swizzle; they must agree with the row table
                const int m = (hdr[0] - (t & ~31)) < 32 ? hdr[0] - (t & ~31) : 32;
                const int sw = (m & 7) == 0 ? 7 : 0;
                const int base = (int)(sroff[r0] & 0xfffu);
                auto Et = [&](int k) { const unsigned r = sroff[r0 + k]; return (int)(r & 0xfffu) + (lane ^ (int)(r >> 12)); };
                auto E = [&](int k) { return base + m * k + (lane ^ (k & sw)); };
                for (int k = 0; k < ns; k++) if (E(k) != Et(k)) return 10;
                for (int k = 0; k < ns; k++) if (E(k) >= ne || sidx[E(k)] >= n) return 5;
                const double c0 = sc0[t];
                auto U = [&](int k) { int i = sidx[E(k)]; return std::make_pair(up[2 * (n0 + i)], up[2 * (n0 + i) + 1]); };
                if (mtype != MEL_MAT_ELASTIC_LINEAR) return 6;   // this model covers the linear elastic pass
                double E11 = 0., E12 = 0., E22 = 0.;
                for (int k = 0; k < ns; k++) {
                    double dx = sp[2 * E(k)], dy = sp[2 * E(k) + 1];
                    auto u = U(k);
                    E11 = E11 + dx * u.first;
                    E12 = E12 + (dx * u.second + dy * u.first);
                    E22 = E22 + dy * u.second;
                }
                E12 = 0.5 * E12;
                double J = 1. + E11 + E22;
                double S33 = Lam * (J - 1.);
                double Mu2 = 2 * Mu;
                double S11 = S33 + Mu2 * E11, S22 = S33 + Mu2 * E22, S12 = Mu2 * E12;
                for (int k = 0; k < ns; k++) {
                    double dx = sp[2 * E(k)], dy = sp[2 * E(k) + 1];
                    sp[2 * E(k)] = c0 * (dx * S11 + dy * S12);
                    sp[2 * E(k) + 1] = c0 * (dy * S22 + dx * S12);
                }
            }
            const uint16_t* stnode = reinterpret_cast<const uint16_t*>(buf.data() + L.tnode);
            for (int t = 0; t < hdr[2]; t++) {
                const uint32_t rec = stn[t];
                const int node = wide ? (int)stnode[t] : (int)(rec & 0xfffu), cnt = (int)((rec >> 12) & 0xffu), pr = (int)(rec >> 20);
                if (wide && (int)(rec & 0xfffu) != (node & 0xfff)) return 12;
                const int lane = t & 31;
                if (node >= n || cnt == 0 || pr + cnt > hdr[3]) return 7;
                // counts descend within a group, so slots with more than j entries are a prefix
                if ((t & 31) && ((int)((stn[t - 1] >> 12) & 0xffu) < cnt || (int)(stn[t - 1] >> 20) != pr)) return 9;
                const int pfull = (t | 31) < hdr[2] ? (int)((stn[t | 31] >> 12) & 0xffu) : 0;
                const int pbase = (int)sroff[pr];
                for (int j = 0; j < pfull && j < cnt; j++) if (pbase + 32 * j != (int)sroff[pr + j]) return 11;
                double fx = sf[2 * node], fy = sf[2 * node + 1];
                for (int j = 0; j < cnt; j++) {
                    const int q = j < pfull ? pbase + 32 * j + lane : (int)sroff[pr + j] + lane;
                    if (q >= ne || stpos[q] >= ne) return 8;
                    fx = fx - sp[2 * stpos[q]];
                    fy = fy - sp[2 * stpos[q] + 1];
                }
                sf[2 * node] = fx; sf[2 * node + 1] = fy;
            }
        }
        for (int i = 0; i < 2 * n; i++) f[2 * n0 + i] = sf[i];
    }
    return 0;
}

// The mixed pass's two-buffer images (pull pieces).  Checks every index the kernel follows and
// the layout's invariants: the pieces list the entries back to back in node order, at most
// MEL_PIECE each, every piece's entries are stored for its node, a node's pieces belong to one
// warp, and every stored entry of a point is listed once.  Then forms FP64 contributions
// c0 * (dN . up) from the stored FP32 derivatives (a stand-in for the kernel's strain and stress,
// enough to exercise the indexing) and returns the nodal sums two ways: f_list piece by piece,
// f_direct by scattering each point's contributions directly.  stats: [chunks, listed entries, largest
// image bytes, largest warp share / mean share x 1000].
extern "C" int emul_segmented_pull(const mel_model_desc* d, int ecap, const double* up, double* f_list,
                                   double* f_direct, long long* stats)
{
    mel_chunk_set CS;
    if (mel_build_chunks(d, ecap, CS, true, 1LL << 62) != MEL_OK) return 100;
    stats[0] = (long long)CS.chunks.size(); stats[1] = 0; stats[2] = CS.img_max; stats[3] = 0;
    memset(f_list, 0, sizeof(double) * 2 * (size_t)d->n_nodes);
    memset(f_direct, 0, sizeof(double) * 2 * (size_t)d->n_nodes);
    for (int b = 0; b < d->n_bodies; b++) {
        if (d->body_type[b] != MEL_BODY_DEFORMABLE) continue;
        if (CS.b_pipe[b]) return 20;
        const int n0 = d->body_node_ptr[b], n = d->body_node_ptr[b + 1] - n0;
        for (int ci = CS.b_chunk0[b]; ci < CS.b_chunk0[b + 1]; ci++) {
            const mel_chunk& c = CS.chunks[ci];
            if (c.bytes % 16 || c.img % 16 || c.bytes > CS.img_max) return 21;
            std::vector<uint8_t> buf(CS.img.begin() + c.img, CS.img.begin() + c.img + c.bytes);
            int hdr[4];
            memcpy(hdr, buf.data(), sizeof hdr);
            if (hdr[0] > MEL_CHUNK_GP_FP64 || hdr[1] % 8 || hdr[1] > ecap || hdr[3] > 1024) return 22;
            const mel_chunk_layout L = mel_chunk_sections(hdr[0], hdr[1], hdr[2], hdr[3], 8);
            if (L.bytes != c.bytes) return 23;
            const float* sp = reinterpret_cast<const float*>(buf.data() + L.dN);
            const uint16_t* sidx = reinterpret_cast<const uint16_t*>(buf.data() + L.idx);
            const uint16_t* spos = reinterpret_cast<const uint16_t*>(buf.data() + L.tpos);
            const double* sc0 = reinterpret_cast<const double*>(buf.data() + L.c0);
            const uint32_t* sgpm = reinterpret_cast<const uint32_t*>(buf.data() + L.gpm);
            const uint16_t* swr = reinterpret_cast<const uint16_t*>(buf.data() + L.tn);
            const uint16_t* ssn = swr + (MEL_PULL_WARPS + 1);
            const uint16_t* sroff = reinterpret_cast<const uint16_t*>(buf.data() + L.roff);
            const int ne = hdr[1];
            // contributions per stored position, and the direct scatter
            std::vector<double> q(2 * (size_t)ne, 0.);
            std::vector<int> listed(ne, 0), stored(ne, 0);
            for (int t = 0; t < hdr[0]; t++) {
                const uint32_t gm = sgpm[t];
                const int r0 = (int)(gm & 0x3ffu), lane = (int)((gm >> 10) & 0x1fu), ns = (int)(gm >> 15);
                if (r0 + ns > hdr[3] || lane != t % 32) return 24;
                const int m = (hdr[0] - (t & ~31)) < 32 ? hdr[0] - (t & ~31) : 32;
                const int sw = (m & 7) == 0 ? 7 : 0;
                const int base = (int)(sroff[r0] & 0xfffu);
                for (int k = 0; k < ns; k++) {
                    const int e = base + m * k + (lane ^ (k & sw));
                    if (e >= ne || sidx[e] >= n) return 25;
                    const int i = sidx[e];
                    const double v = (double)sp[2 * e] * up[2 * (n0 + i)] + (double)sp[2 * e + 1] * up[2 * (n0 + i) + 1];
                    q[2 * e] = sc0[t] * v;
                    q[2 * e + 1] = sc0[t] * (v + (double)sp[2 * e]);
                    stored[e]++;
                    f_direct[2 * (n0 + i)] -= q[2 * e];
                    f_direct[2 * (n0 + i) + 1] -= q[2 * e + 1];
                }
            }
            // pieces: (first listed entry, count, node); the listed entries, in order, are the
            // pieces' entries back to back
            const uint32_t* spc = reinterpret_cast<const uint32_t*>(buf.data() + L.tn + 16);
            const int npc = swr[MEL_PULL_WARPS];
            if (swr[0] != 0 || 16 + 4 * npc > 4 * ((hdr[2] + 3) & ~3)) return 26;
            int nl = 0, share_max = 0, prev_node = -1, prev_warp = -1;
            for (int w = 0; w < MEL_PULL_WARPS; w++) {
                const int a = swr[w], e1 = swr[w + 1];
                if (e1 < a || e1 > npc) return 27;
                int share = 0;
                for (int pi = a; pi < e1; pi++) {
                    const uint32_t rec = spc[pi];
                    const int q0 = (int)(rec & 0x1fffu), cnt = (int)((rec >> 13) & 7u) + 1, node = (int)((rec >> 16) & 0xffffu);
                    if (q0 != nl || cnt > MEL_PIECE || node >= n) return 28;
                    if (node < prev_node) return 31;                           // sorted by node
                    if (node == prev_node && w != prev_warp) return 33;        // a node within one warp
                    double sx = 0., sy = 0.;
                    for (int i = 0; i < cnt; i++) {
                        const int qq = q0 + i;
                        if (qq >= ne || spos[qq] >= ne) return 29;
                        if (sidx[spos[qq]] != node) return 30;                 // listed node is the stored one
                        listed[spos[qq]]++;
                        sx += q[2 * spos[qq]];
                        sy += q[2 * spos[qq] + 1];
                    }
                    f_list[2 * (n0 + node)] -= sx;
                    f_list[2 * (n0 + node) + 1] -= sy;
                    nl += cnt;
                    share += cnt;
                    prev_node = node;
                    prev_warp = w;
                }
                share_max = std::max(share_max, share);
            }
            stats[1] += nl;
            for (int e = 0; e < ne; e++) if (listed[e] != stored[e]) return 32;   // each stored entry once
            if (nl > 0) stats[3] = std::max(stats[3], (long long)share_max * 1000 * MEL_PULL_WARPS / nl);
        }
    }
    return 0;
}
