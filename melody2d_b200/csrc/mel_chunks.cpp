// Host builder of the chunk images (layout in mel_internal.h).  Points are cut into chunks in
// index order; within a chunk they are stored row by row in groups of up to 32 slots sorted by
// support count, and the pull records list, for every touched node, the positions of its entries
// in ascending Gauss-point order (the order Body::Update_internal_forces accumulates them in,
// Code/Body.h:960-1050), in rows of up to 32 nodes sorted by entry count.
#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <numeric>
#include "mel_chunks.h"

void mel_set_error(const char* fmt, ...);

namespace {

// slots of a chunk whose points have supports ns[0..n): slot order and per-group row tables
struct slot_plan {
    std::vector<int> order;      // point offsets within the chunk, in slot order
    std::vector<int> first_row;  // per slot: start of its group's row table in roff
    std::vector<int> lane;       // per slot: lane within its group
    std::vector<int> roff;       // row tables: entry offset of row k of a group
    std::vector<int> rsw;        // per row: lane swizzle (XOR, 0..7)
    int entries = 0;
    // stored position of entry k of slot s
    int pos(int s, int k) const { const int r = first_row[s] + k; return roff[r] + (lane[s] ^ rsw[r]); }
};

slot_plan plan_slots(const int* ns, int n)
{
    slot_plan P;
    P.order.resize(n);
    std::iota(P.order.begin(), P.order.end(), 0);
    std::stable_sort(P.order.begin(), P.order.end(), [&](int a, int b) { return ns[a] > ns[b]; });
    P.first_row.resize(n);
    P.lane.resize(n);
    for (int s0 = 0; s0 < n; s0 += 32) {
        const int m = std::min(32, n - s0);
        const int K = ns[P.order[s0]];
        const int r0 = (int)P.roff.size();
        for (int j = 0; j < m; j++) { P.first_row[s0 + j] = r0; P.lane[s0 + j] = j; }
        for (int k = 0; k < K; k++) {
            // every row of a group is m wide: slots with fewer supports are padded (zero
            // derivatives, node 0), so that entry k of lane j sits at base + m k + (j ^ swizzle)
            // and the kernel computes every position instead of reading a row table
            P.roff.push_back(P.entries);
            // rows whose width is a multiple of 8 rotate the lanes' bank groups from row to row
            // (lane ^ (k & 7) stays inside its aligned block of 8, so the row stays a permutation
            // of consecutive entries); otherwise all entries of a point would share one bank
            // group, and the pull, whose lanes read entries of points shared by nearby nodes,
            // would meet them in the same bank
            P.rsw.push_back(m % 8 == 0 ? (k & 7) : 0);
            P.entries += m;
        }
    }
    return P;
}

// stored entries of points with supports ns[0..n) once the groups are padded to their widest slot
int padded_entries(const int* ns, int n)
{
    std::vector<int> v(ns, ns + n);
    std::sort(v.begin(), v.end(), std::greater<int>());
    int e = 0;
    for (int s0 = 0; s0 < n; s0 += 32) e += std::min(32, n - s0) * v[s0];
    return e;
}

// rows of all row tables of points with supports ns[0..n)
int table_rows(const int* ns, int n)
{
    int rows = 0;
    std::vector<int> v(ns, ns + n);
    std::sort(v.begin(), v.end(), std::greater<int>());
    for (int s0 = 0; s0 < n; s0 += 32) rows += v[s0];
    return rows;
}

}  // namespace

long long mel_body_entries(const mel_model_desc* d, int b)
{
    return (long long)d->gp_sup_ptr[d->body_gp_ptr[b + 1]] - d->gp_sup_ptr[d->body_gp_ptr[b]];
}

mel_status mel_build_chunks(const mel_model_desc* d, int ecap, mel_chunk_set& out, bool mixed, long long pipe_min_entries)
{
    const int nb = d->n_bodies;
    out.b_pipe.assign(nb, 0);
    out.chunks.clear();
    out.img.clear();
    out.b_chunk0.assign(nb + 1, 0);
    out.img_max = 16;
    out.n_entries = 0;
    out.n_pad = 0;
    std::vector<int> ns;
    std::vector<std::pair<long long, int>> tp;   // (node << 32 | point, stored position)
    for (int b = 0; b < nb; b++) {
        out.b_chunk0[b] = (int)out.chunks.size();
        if (d->body_type[b] != MEL_BODY_DEFORMABLE) continue;
        const int nnb = d->body_node_ptr[b + 1] - d->body_node_ptr[b];
        if (nnb > MEL_MAX_WIDE_NODES) { mel_set_error("deformable body %d has %d nodes (16-bit node indices: at most %d)", b, nnb, MEL_MAX_WIDE_NODES); return MEL_ERR_UNSUPPORTED; }
        // a body above MEL_MAX_BODY_NODES nodes: its FP64 pull slots name their node in a 16-bit
        // section (the records hold 12 bits), and it never runs the mixed pipeline
        const int wide = nnb > MEL_MAX_BODY_NODES ? 1 : 0;
        int g = d->body_gp_ptr[b];
        const int g1 = d->body_gp_ptr[b + 1];
        const bool pipe = mixed && !wide && mel_body_entries(d, b) >= pipe_min_entries;
        out.b_pipe[b] = pipe ? 1 : 0;
        const int gpcap = pipe ? MEL_CHUNK_GP_MX : MEL_CHUNK_GP_FP64;
        while (g < g1) {
            // as many points as fit gpcap slots (one point thread each), ecap entries and the 10-bit
            // row tables
            int ngp = 0, nent = 0, nsmax = 0;
            ns.clear();
            while (g + ngp < g1 && ngp < gpcap) {
                int c = d->gp_sup_ptr[g + ngp + 1] - d->gp_sup_ptr[g + ngp];
                if (c > 255 || c <= 0) { mel_set_error("Gauss point %d has %d supports (1..255 supported)", g + ngp, c); return MEL_ERR_UNSUPPORTED; }
                if (nent + c > ecap) break;
                ns.push_back(c);
                if (padded_entries(ns.data(), ngp + 1) > ecap) { ns.pop_back(); break; }
                nsmax = std::max(nsmax, c);
                // row tables are addressed with 10 bits; the exact count is needed only when the
                // bound (groups x largest count) could exceed that
                if (((ngp + 32) / 32) * nsmax > 1023 && table_rows(ns.data(), ngp + 1) > 1023) { ns.pop_back(); break; }
                nent += c;
                ngp++;
            }
            if (ngp == 0) { mel_set_error("Gauss point %d has more supports than a chunk holds", g); return MEL_ERR_UNSUPPORTED; }
            if (nent > 4096) { mel_set_error("chunk entry cap %d above 4096", ecap); return MEL_ERR_INVALID; }
            const slot_plan P = plan_slots(ns.data(), ngp);
            mel_chunk ch;
            memset(&ch, 0, sizeof ch);
            ch.gp0 = g;
            ch.ngp = ngp;
            ch.ne = (P.entries + 7) & ~7;
            // stored position of every entry; pull order by (node, point index)
            tp.clear();
            for (int slot = 0; slot < ngp; slot++) {
                const int t = P.order[slot];
                const int gg = g + t;
                for (int k = 0, j = d->gp_sup_ptr[gg]; j < d->gp_sup_ptr[gg + 1]; k++, j++) {
                    int v = d->gp_sup_idx[j];
                    if (v < 0 || v >= nnb) { mel_set_error("Gauss support index out of range"); return MEL_ERR_INVALID; }
                    tp.push_back({ ((long long)v << 32) | (long long)t, P.pos(slot, k) });
                }
            }
            std::sort(tp.begin(), tp.end());
            if (mixed && !pipe) {
                // pull of the mixed two-buffer loop: the entries in (node, point) order with their
                // stored positions, cut into pieces of at most MEL_PIECE entries of one node, and the
                // seven pull warps' ranges of pieces cut at node boundaries (every node belongs to
                // one warp), balanced by entries
                const int nent_l = (int)tp.size();
                std::vector<uint32_t> pcs;
                std::vector<int> pc_first;                       // first piece of each node run
                for (int q = 0; q < nent_l;) {
                    int r = q;
                    while (r < nent_l && (tp[r].first >> 32) == (tp[q].first >> 32)) r++;
                    const int len = r - q, np = (len + MEL_PIECE - 1) / MEL_PIECE;
                    pc_first.push_back((int)pcs.size());
                    for (int k = 0, at = q; k < np; k++) {
                        const int c = len / np + (k < len % np ? 1 : 0);
                        pcs.push_back((uint32_t)at | ((uint32_t)(c - 1) << 13) | ((uint32_t)(tp[q].first >> 32) << 16));   // node: 16 bits
                        at += c;
                    }
                    q = r;
                }
                const int npc = (int)pcs.size();
                pc_first.push_back(npc);
                const int segw = (2 * (MEL_PULL_WARPS + 1) + 4 * npc + 3) / 4 + 1;
                ch.ntn = segw;
                const int nroff = (int)P.roff.size();
                if (nroff > 4095) { mel_set_error("chunk row tables too large (%d rows)", nroff); return MEL_ERR_UNSUPPORTED; }
                const mel_chunk_layout L = mel_chunk_sections(ch.ngp, ch.ne, segw, nroff, 8);
                ch.bytes = L.bytes;
                ch.img = (long long)out.img.size();
                out.img.resize(out.img.size() + L.bytes, 0);
                uint8_t* I = out.img.data() + ch.img;
                int hdr[4] = { ch.ngp, ch.ne, segw, nroff };
                memcpy(I, hdr, sizeof hdr);
                float* dNf = reinterpret_cast<float*>(I + L.dN);
                uint16_t* idx = reinterpret_cast<uint16_t*>(I + L.idx);
                uint16_t* spos = reinterpret_cast<uint16_t*>(I + L.tpos);
                double* c0 = reinterpret_cast<double*>(I + L.c0);
                uint32_t* gpm = reinterpret_cast<uint32_t*>(I + L.gpm);
                uint16_t* wr = reinterpret_cast<uint16_t*>(I + L.tn);       // MEL_PULL_WARPS + 1 bounds
                uint32_t* pcr = reinterpret_cast<uint32_t*>(I + L.tn + 16);  // piece records
                uint16_t* roff = reinterpret_cast<uint16_t*>(I + L.roff);
                for (int slot = 0; slot < ngp; slot++) {
                    const int gg = g + P.order[slot];
                    const int c = d->gp_sup_ptr[gg + 1] - d->gp_sup_ptr[gg];
                    c0[slot] = d->gp_weight[gg] * d->gp_jacobian[gg];   // c0 of Code/Body.h:994
                    gpm[slot] = (uint32_t)P.first_row[slot] | ((uint32_t)P.lane[slot] << 10) | ((uint32_t)c << 15);
                    for (int k = 0, j = d->gp_sup_ptr[gg]; k < c; k++, j++) {
                        const int e = P.pos(slot, k);
                        idx[e] = (uint16_t)d->gp_sup_idx[j];
                        dNf[2 * e] = (float)d->gp_dNdx[j];
                        dNf[2 * e + 1] = (float)d->gp_dNdy[j];
                    }
                }
                for (int q = 0; q < nent_l; q++) spos[q] = (uint16_t)tp[q].second;
                for (int k = 0; k < npc; k++) pcr[k] = pcs[k];
                // warp w takes the pieces [wr[w], wr[w+1]): cut at the node boundary whose entry
                // offset is nearest to w/7 of the entries
                const int nruns = (int)pc_first.size() - 1;
                std::vector<int> run_at(nruns + 1, nent_l);      // first entry of each node run
                for (int r = 0; r < nruns; r++) run_at[r] = (int)(pcs[pc_first[r]] & 0x1fffu);
                wr[0] = 0;
                int r = 0;
                for (int w = 1; w < MEL_PULL_WARPS; w++) {
                    const long long target = ((long long)w * nent_l) / MEL_PULL_WARPS;
                    while (r < nruns && std::llabs(run_at[r + 1] - target) <= std::llabs(run_at[r] - target)) r++;
                    wr[w] = (uint16_t)pc_first[r];
                }
                wr[MEL_PULL_WARPS] = (uint16_t)npc;
                for (int r = 0; r < nroff; r++) roff[r] = (uint16_t)(P.roff[r] | (P.rsw[r] << 12));
                out.img_max = std::max(out.img_max, ch.bytes);
                out.n_entries += ch.ne;
                out.n_pad += ch.ne - nent;
                out.chunks.push_back(ch);
                g += ngp;
                continue;
            }
            // touched nodes: (first entry in tp, count), then pull slots sorted by count
            std::vector<std::pair<int, int>> tnodes;
            for (int q = 0; q < (int)tp.size(); q++)
                if (q == 0 || (tp[q].first >> 32) != (tp[q - 1].first >> 32)) tnodes.push_back({ q, 1 });
                else tnodes.back().second++;
            std::stable_sort(tnodes.begin(), tnodes.end(),
                             [](const std::pair<int, int>& a, const std::pair<int, int>& b) { return a.second > b.second; });
            ch.ntn = (int)tnodes.size();
            // pull row tables after the point groups' rows: row j of a pull group holds entry j of
            // every slot with more than j entries (a prefix of the group)
            std::vector<int> roff_all(P.roff);
            std::vector<int> rsw_all(P.rsw);
            std::vector<uint32_t> tn(ch.ntn);
            std::vector<uint16_t> tnv(ch.ntn);
            std::vector<uint16_t> tposv(P.entries);
            int pe = 0;
            for (int s0 = 0; s0 < ch.ntn; s0 += 32) {
                const int m = std::min(32, ch.ntn - s0);
                const int K = tnodes[s0].second;
                const int r0 = (int)roff_all.size();
                for (int j = 0; j < K; j++) {
                    roff_all.push_back(pe);
                    rsw_all.push_back(0);
                    int mj = 0;
                    while (mj < m && tnodes[s0 + mj].second > j) mj++;
                    for (int l = 0; l < mj; l++) tposv[pe + l] = (uint16_t)tp[tnodes[s0 + l].first + j].second;
                    pe += mj;
                }
                for (int l = 0; l < m; l++) {
                    const int node = (int)(tp[tnodes[s0 + l].first].first >> 32);
                    tn[s0 + l] = (uint32_t)(node & 0xfff) | ((uint32_t)tnodes[s0 + l].second << 12) | ((uint32_t)r0 << 20);
                    tnv[s0 + l] = (uint16_t)node;
                }
            }
            const int nroff = (int)roff_all.size();
            if (nroff > 4095 || pe != nent) {
                mel_set_error("chunk row tables too large (%d rows)", nroff);
                return MEL_ERR_UNSUPPORTED;
            }
            const int wsec = (wide && !mixed) ? 1 : 0;     // the mixed pipeline is off for wide bodies
            const mel_chunk_layout L = mel_chunk_sections(ch.ngp, ch.ne, ch.ntn, nroff, mixed ? 8 : 16, wsec);
            ch.bytes = L.bytes;
            ch.img = (long long)out.img.size();
            out.img.resize(out.img.size() + L.bytes, 0);
            uint8_t* I = out.img.data() + ch.img;
            int hdr[4] = { ch.ngp, ch.ne, ch.ntn, nroff };
            memcpy(I, hdr, sizeof hdr);
            double* dN = reinterpret_cast<double*>(I + L.dN);
            float* dNf = reinterpret_cast<float*>(I + L.dN);
            uint16_t* idx = reinterpret_cast<uint16_t*>(I + L.idx);
            uint16_t* tpos = reinterpret_cast<uint16_t*>(I + L.tpos);
            double* c0 = reinterpret_cast<double*>(I + L.c0);
            uint32_t* gpm = reinterpret_cast<uint32_t*>(I + L.gpm);
            uint32_t* tnr = reinterpret_cast<uint32_t*>(I + L.tn);
            uint16_t* roff = reinterpret_cast<uint16_t*>(I + L.roff);
            for (int slot = 0; slot < ngp; slot++) {
                const int gg = g + P.order[slot];
                const int c = d->gp_sup_ptr[gg + 1] - d->gp_sup_ptr[gg];
                c0[slot] = d->gp_weight[gg] * d->gp_jacobian[gg];   // c0 of Code/Body.h:994
                gpm[slot] = (uint32_t)P.first_row[slot] | ((uint32_t)P.lane[slot] << 10) | ((uint32_t)c << 15);
                for (int k = 0, j = d->gp_sup_ptr[gg]; k < c; k++, j++) {
                    int e = P.pos(slot, k);
                    idx[e] = (uint16_t)d->gp_sup_idx[j];
                    if (mixed) { dNf[2 * e] = (float)d->gp_dNdx[j]; dNf[2 * e + 1] = (float)d->gp_dNdy[j]; }
                    else { dN[2 * e] = d->gp_dNdx[j]; dN[2 * e + 1] = d->gp_dNdy[j]; }
                }
            }
            for (int q = 0; q < P.entries; q++) tpos[q] = tposv[q];
            memcpy(tnr, tn.data(), sizeof(uint32_t) * tn.size());
            if (wsec) memcpy(I + L.tnode, tnv.data(), sizeof(uint16_t) * tnv.size());
            for (int r = 0; r < nroff; r++) roff[r] = (uint16_t)(roff_all[r] | (rsw_all[r] << 12));
            out.img_max = std::max(out.img_max, ch.bytes);
            out.n_entries += ch.ne;
            out.n_pad += ch.ne - nent;
            out.chunks.push_back(ch);
            g += ngp;
        }
    }
    out.b_chunk0[nb] = (int)out.chunks.size();
    return MEL_OK;
}
