// Host side of the B200 solver: builds the device-resident model from a mel_model_desc, runs the
// set-up of Code/main.cpp:104-127, advances the step loop of Code/main.cpp:141-196 and implements
// the C ABI declared in include/melgpu.h.
#include <cstdarg>
#include <cstdlib>
#include <cstdio>
#include <cstring>
#include <cmath>
#include <string>
#include <numeric>
#include <vector>
#include <algorithm>
#include <fstream>
#include <iomanip>
#include "mel_internal.h"
#include "mel_prox_host.h"
#include "mel_chunks.h"
#include "mel_material.h"
#include "mel_host.h"   // .asc loader (mel_loader.cpp)
#include "mel_sincos.h"

// ---------------------------------------------------------------------------------------------
// errors
// ---------------------------------------------------------------------------------------------
static thread_local std::string g_err;
void mel_set_error(const char* fmt, ...)
{
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    g_err = buf;
}
void mel_set_cuda_error(cudaError_t e, const char* what, const char* file, int line)
{
    mel_set_error("CUDA error %s (%s) in %s at %s:%d", cudaGetErrorName(e), cudaGetErrorString(e), what, file, line);
}

// ---------------------------------------------------------------------------------------------
// handle
// ---------------------------------------------------------------------------------------------
// asynchronous checkpoint (mel_checkpoint_start / mel_checkpoint_read)
struct mel_ckpt {
    cudaStream_t side = nullptr;        // device-to-host copies, off the solver's stream
    cudaEvent_t packed = nullptr;       // snapshot taken on the solver's stream
    cudaEvent_t landed = nullptr;       // snapshot in pinned host memory
    char* d_stage = nullptr; size_t d_cap = 0;
    char* h_stage = nullptr; size_t h_cap = 0;
    bool pending = false;
    int nn = 0, nb = 0, ncont = 0;
    double time = 0., dt = 0., next_cup = 0.;
};

struct mel_handle {
    mel_dev d;
    mel_prox_state P;
    mel_prox_host H;
    cudaStream_t stream = nullptr;
    int device = 0;
    std::vector<void*> allocs;
    // host mirrors
    int nb = 0, nn = 0, nbd = 0, ne = 0, ng = 0, nge = 0, nse = 0;
    std::vector<int> b_type, b_status, b_node0, b_mat;
    std::vector<double> X0, rg_file, rg_mat;
    double time = 0., dt = 0., cup = 0., next_cup = 0.;
    mel_ckpt ck;
    int solver = 0;
    int flags[MEL_NFLAGS] = { 0 };
    int parity = 0;
    size_t body_smem = 0;
    int nblocks_body = 0;     // body-kernel CTAs, and the wide bodies' CTAs after them
    int nwide = 0;
    int chunk_cap = 0;          // support entries per chunk chosen at build time
    int body_stages = 2;        // image buffers per CTA (3 when a body runs the mixed pipeline)
    double img_bytes = 0.;      // bytes of all chunk images
    long long n_pad = 0;        // padding entries in the chunk images
    int launches = 0;
    double t_contact = 0., t_body = 0., t_prox = 0.;
    int timing = 0;
    double* d_monitor = nullptr;
    double* d_monitor_part = nullptr;
    double* d_state = nullptr;   // node state in the 12-doubles-per-node layout (mel_get/set_node_state)
    // border contact pressures: 0 = up to date, 1 = the last step's, still computable from the
    // current contact list, 2 = that list was replaced by a proximity update since (batch member
    // without recording)
    int pressure_state = 0;
    // Solver_step: Body::Store snapshot (device), time of the last Update_bc, statistics of the
    // last step {neval, max_error, mean_error, total_mass, max_mass}, reduction output (pinned)
    std::vector<void*> store_bufs;
    size_t store_cont_cap = 0;
    int store_ncont = 0;
    double t_bc = 0.;
    double solver_stats[5] = { 0., 0., 0., 0., 0. };
    double* h_red = nullptr;
    double* d_red = nullptr;
    int* d_rigid_ids = nullptr;
    int nrigid = 0;
    int precision = MEL_PREC_FP64;
    double t_total = 0.;
    cudaEvent_t ev_start = nullptr, ev_end = nullptr;
    std::vector<cudaEvent_t> ev_pool;
    double bytes_body = 0., bytes_contact = 0.;
    int n_def_nodes = 0;
    // Monitoring on the device (mel_monitor_setup): entries, per-body partial sums, row buffer of
    // mon_cap rows of mon_stride doubles, rows recorded since the last drain, Number_iteration
    mel_mon_op* mon_ops = nullptr;
    int mon_nops = 0, mon_energy = 0, mon_bound = 0;
    double* mon_part = nullptr;
    double* mon_rows = nullptr;
    int mon_cap = 0, mon_stride = 0, mon_count = 0;
    bool mon_on = false, mon_forces = false;
    // DEACTIVATION entries (device copy) that Update_status evaluates after each proximity update
    double* d_deact = nullptr;
    int n_deact = 0;
    bool deact_forces = false;
    long long iteration = 0;
    mel_batch* batch = nullptr;  // batch the handle is a member of (steps only through the batch)
    int failed = 0;                 // model-level failure (MEL_ERR_NAN, MEL_ERR_BOUNDS) that retired it from a batch
    std::string failed_msg;
};

template <typename T>
static T* dalloc(mel_handle* h, size_t n)
{
    void* p = nullptr;
    if (n == 0) n = 1;
    if (cudaMalloc(&p, n * sizeof(T)) != cudaSuccess) return nullptr;
    cudaMemset(p, 0, n * sizeof(T));
    h->allocs.push_back(p);
    return (T*)p;
}
template <typename T>
static T* dupload(mel_handle* h, const T* src, size_t n)
{
    T* p = dalloc<T>(h, n);
    if (p && src && n) cudaMemcpy(p, src, n * sizeof(T), cudaMemcpyHostToDevice);
    return p;
}
template <typename T>
static T* dupload(mel_handle* h, const std::vector<T>& v) { return dupload(h, v.data(), v.size()); }

// ---------------------------------------------------------------------------------------------
// host restatements of set-up functions
// ---------------------------------------------------------------------------------------------
// Body::Initialize_segments (Code/Body.h:403-606): segment node tables and initial lengths
static void initialize_segments(const mel_model_desc* d, int b, std::vector<int>& sn, std::vector<int>& ss,
                                std::vector<double>& len0)
{
    double period = d->period[1] - d->period[0];
    int n0 = d->body_node_ptr[b];
    for (int gi = d->body_border_ptr[b]; gi < d->body_border_ptr[b + 1]; gi++) {
        int i = gi - d->body_border_ptr[b];
        int off = d->border_node_ptr[gi];
        int nbn = d->border_node_ptr[gi + 1] - off;
        const int* bn = d->border_nodes + off;
        int gb = d->body_border_ptr[b] + d->border_before[gi];
        int ga = d->body_border_ptr[b] + d->border_after[gi];
        const int* bnb = d->border_nodes + d->border_node_ptr[gb];
        int nbb = d->border_node_ptr[gb + 1] - d->border_node_ptr[gb];
        const int* bna = d->border_nodes + d->border_node_ptr[ga];
        int per = d->border_periodicity[gi];
        auto N = [&](int k, int j) -> int& { return sn[4 * (off + j) + k]; };
        auto S = [&](int k, int j) -> int& { return ss[4 * (off + j) + k]; };
        N(0, 0) = bnb[nbb - 2]; N(1, 0) = bn[0]; N(2, 0) = bn[1]; N(3, 0) = bn[2];
        if (per == MEL_PER_PERIODIC && i == 0) S(0, 0) = -1;
        else if (per == MEL_PER_PERIODIC) S(0, 0) = 1;
        for (int j = 1; j < nbn - 2; j++) { N(0, j) = bn[j - 1]; N(1, j) = bn[j]; N(2, j) = bn[j + 1]; N(3, j) = bn[j + 2]; }
        N(0, nbn - 2) = bn[nbn - 3]; N(1, nbn - 2) = bn[nbn - 2]; N(2, nbn - 2) = bn[nbn - 1]; N(3, nbn - 2) = bna[1];
        if (per == MEL_PER_PERIODIC && i == 0) { S(2, nbn - 2) = 1; S(3, nbn - 2) = 1; }
        else if (per == MEL_PER_PERIODIC) { S(2, nbn - 2) = -1; S(3, nbn - 2) = -1; }
        N(0, nbn - 1) = bn[nbn - 2]; N(1, nbn - 1) = bn[nbn - 1]; N(2, nbn - 1) = bna[1]; N(3, nbn - 1) = bna[2];
        if (per == MEL_PER_PERIODIC) {
            int s = (i == 0) ? 1 : -1;
            S(1, nbn - 1) = s; S(2, nbn - 1) = s; S(3, nbn - 1) = s;
        }
        for (int j = 0; j < nbn; j++) {
            const double* X = d->node_x0;
            double x0 = X[2 * (n0 + N(0, j))] + S(0, j) * period, y0 = X[2 * (n0 + N(0, j)) + 1];
            double x1 = X[2 * (n0 + N(1, j))] + S(1, j) * period, y1 = X[2 * (n0 + N(1, j)) + 1];
            double x2 = X[2 * (n0 + N(2, j))] + S(2, j) * period, y2 = X[2 * (n0 + N(2, j)) + 1];
            len0[off + j] = 0.5 * sqrt((x1 - x0) * (x1 - x0) + (y1 - y0) * (y1 - y0)) + 0.5 * sqrt((x2 - x1) * (x2 - x1) + (y2 - y1) * (y2 - y1));
        }
    }
}

static double tri_surface(double x0, double y0, double x1, double y1, double x2, double y2)
{   // Code/Tools.h:377-380
    return 0.5 * fabs((x1 - x0) * (y2 - y0) - (x2 - x0) * (y1 - y0));
}
static double tri_inertia(double x0, double y0, double x1, double y1, double x2, double y2, double xc, double yc)
{   // Code/Tools.h:388-412
    double a, PP, PQ, QQ, I = 0;
    a = tri_surface(xc, yc, x0, y0, x1, y1);
    PP = (x0 - xc) * (x0 - xc) + (y0 - yc) * (y0 - yc); PQ = (x0 - xc) * (x1 - xc) + (y0 - yc) * (y1 - yc); QQ = (x1 - xc) * (x1 - xc) + (y1 - yc) * (y1 - yc);
    I += a * (PP + PQ + QQ);
    a = tri_surface(xc, yc, x1, y1, x2, y2);
    PP = (x1 - xc) * (x1 - xc) + (y1 - yc) * (y1 - yc); PQ = (x1 - xc) * (x2 - xc) + (y1 - yc) * (y2 - yc); QQ = (x2 - xc) * (x2 - xc) + (y2 - yc) * (y2 - yc);
    I += a * (PP + PQ + QQ);
    a = tri_surface(xc, yc, x2, y2, x0, y0);
    PP = (x2 - xc) * (x2 - xc) + (y2 - yc) * (y2 - yc); PQ = (x2 - xc) * (x0 - xc) + (y2 - yc) * (y0 - yc); QQ = (x0 - xc) * (x0 - xc) + (y0 - yc) * (y0 - yc);
    I += a * (PP + PQ + QQ);
    return fabs(I / 6.);
}

// ---------------------------------------------------------------------------------------------
// construction
// ---------------------------------------------------------------------------------------------
static mel_status validate(const mel_model_desc* d)
{
    if (!d) { mel_set_error("null model description"); return MEL_ERR_INVALID; }
    if (d->abi_version != MELGPU_ABI_VERSION) { mel_set_error("abi_version %d, library %d", d->abi_version, MELGPU_ABI_VERSION); return MEL_ERR_INVALID; }
    if (d->n_bodies <= 0 || d->n_nodes <= 0 || d->n_borders <= 0) { mel_set_error("empty model"); return MEL_ERR_INVALID; }
    if (!(d->period[1] > d->period[0])) { mel_set_error("PERIODIC_BOUNDARIES must satisfy Xmin < Xmax"); return MEL_ERR_INVALID; }
    if (!(d->dt > 0.)) { mel_set_error("time step must be positive"); return MEL_ERR_INVALID; }
    if (d->solver < MEL_SOLVER_EULER || d->solver > MEL_SOLVER_EULER_2) { mel_set_error("unknown solver %d", d->solver); return MEL_ERR_INVALID; }
    if (d->body_node_ptr[d->n_bodies] != d->n_nodes) { mel_set_error("body_node_ptr does not cover n_nodes"); return MEL_ERR_INVALID; }
    if (d->body_border_ptr[d->n_bodies] != d->n_borders) { mel_set_error("body_border_ptr does not cover n_borders"); return MEL_ERR_INVALID; }
    for (int g = 0; g < d->n_borders; g++) {
        int nbn = d->border_node_ptr[g + 1] - d->border_node_ptr[g];
        if (nbn < 3) { mel_set_error("border %d has %d nodes (need >= 3)", g, nbn); return MEL_ERR_INVALID; }
        if (d->border_interpolant[g] != MEL_INTERP_LINEAR) { mel_set_error("border %d: Spline interpolant is not supported on the GPU path", g); return MEL_ERR_UNSUPPORTED; }
        int b = d->border_body[g];
        int nnb = d->body_node_ptr[b + 1] - d->body_node_ptr[b];
        for (int k = d->border_node_ptr[g]; k < d->border_node_ptr[g + 1]; k++)
            if (d->border_nodes[k] < 0 || d->border_nodes[k] >= nnb) { mel_set_error("border %d node index out of range", g); return MEL_ERR_INVALID; }
    }
    for (int b = 0; b < d->n_bodies; b++) {
        int nnb = d->body_node_ptr[b + 1] - d->body_node_ptr[b];
        if (d->body_type[b] == MEL_BODY_DEFORMABLE && nnb > MEL_MAX_WIDE_NODES) {
            mel_set_error("deformable body %d has %d nodes; this build indexes at most %d nodes of a body (16 bits)", b, nnb, MEL_MAX_WIDE_NODES);
            return MEL_ERR_UNSUPPORTED;
        }
        if (d->body_material[b] < 0 || d->body_material[b] >= d->n_materials) { mel_set_error("body %d material out of range", b); return MEL_ERR_INVALID; }
    }
    if (d->n_matrix > 0) {
        if (!d->body_matrix_ptr || d->body_matrix_ptr[d->n_bodies] != d->n_matrix) { mel_set_error("body_matrix_ptr does not cover the matrix entries"); return MEL_ERR_INVALID; }
        for (int b = 0; b < d->n_bodies; b++) {
            const int nd = 2 * (d->body_node_ptr[b + 1] - d->body_node_ptr[b]);
            for (int i = d->body_matrix_ptr[b]; i < d->body_matrix_ptr[b + 1]; i++)
                if (d->matrix_dofs[2 * i] < 0 || d->matrix_dofs[2 * i] >= nd || d->matrix_dofs[2 * i + 1] < 0 || d->matrix_dofs[2 * i + 1] >= nd) {
                    mel_set_error("matrix entry %d of body %d names a degree of freedom outside the body", i, b);
                    return MEL_ERR_INVALID;
                }
        }
    }
    return MEL_OK;
}

// Chunk entry cap for a model of this precision whose largest deformable body has max_nodes
// nodes: MELGPU_CHUNK_CAP if set, else the first line of the tuning table (the file named by
// MELGPU_TUNE_FILE; lines "precision max_body_nodes cap", '#' comments) whose precision matches and
// whose node bound covers max_nodes; 0 when neither applies.
static int tuned_chunk_cap(int precision, int max_nodes)
{
    if (const char* c = getenv("MELGPU_CHUNK_CAP")) {
        const int v = atoi(c);
        if (v >= 64 && v <= (precision == MEL_PREC_MIXED ? MEL_CHUNK_E_MAX_MX : MEL_CHUNK_E_MAX)) return v & ~7;
    }
    const char* path = getenv("MELGPU_TUNE_FILE");
    if (!path) return 0;
    FILE* f = fopen(path, "r");
    if (!f) return 0;
    char line[256];
    int cap = 0;
    while (fgets(line, sizeof line, f)) {
        if (line[0] == '#') continue;
        int p = -1, mn = 0, c = 0;
        if (sscanf(line, "%d %d %d", &p, &mn, &c) == 3 && p == precision && max_nodes <= mn && c >= 64 &&
            c <= (precision == MEL_PREC_MIXED ? MEL_CHUNK_E_MAX_MX : MEL_CHUNK_E_MAX)) {
            cap = c & ~7;
            break;
        }
    }
    fclose(f);
    return cap;
}

static mel_status build(mel_handle* h, const mel_model_desc* d, const mel_options* opt)
{
    mel_dev& D = h->d;
    memset(&D, 0, sizeof D);
    h->nb = d->n_bodies; h->nn = d->n_nodes; h->nbd = d->n_borders;
    h->ne = d->border_node_ptr[d->n_borders];
    h->ng = d->n_gauss;
    h->time = d->time; h->dt = d->dt; h->cup = d->contact_update_period; h->next_cup = d->next_contact_update;
    h->solver = d->solver;
    memcpy(h->flags, d->flags, sizeof h->flags);
    h->precision = opt ? opt->precision : MEL_PREC_FP64;
    const int nb = h->nb, nn = h->nn, nbd = h->nbd, ne = h->ne;
    D.nb = nb; D.nn = nn; D.nbd = nbd; D.ne = ne; D.ng = h->ng;
    D.nmat = d->n_materials;
    D.self_contact = (d->flags[8] == 0);
    D.xmin = d->period[0]; D.period = d->period[1] - d->period[0];
    D.gx = d->gravity[0]; D.gy = d->gravity[1];
    D.precision = h->precision;
    D.wait_ns = MEL_WAIT_NS;
    if (const char* w = getenv("MELGPU_WAIT_NS")) {       // test knob: shorter pipeline waits
        char* end = nullptr;
        const unsigned long long v = strtoull(w, &end, 10);
        if (end && *end == 0 && v < MEL_WAIT_NS) D.wait_ns = v;
    }
    // time
    double t2[2] = { d->time, d->time };
    D.time2 = dupload(h, t2, 2);
    D.dt = dupload(h, &d->dt, 1);
    // materials, laws
    D.mat_type = dupload(h, d->material_type, d->n_materials);
    D.mat_p = dupload(h, d->material_params, (size_t)d->n_materials * MEL_MAT_NPARAM);
    D.law_type = dupload(h, d->law_type, d->n_laws);
    D.law_len = dupload(h, d->law_length, d->n_laws);
    D.law_p = dupload(h, d->law_params, (size_t)d->n_laws * MEL_LAW_NPARAM);
    D.table = dupload(h, d->contacts_table, (size_t)d->n_materials * d->n_materials);
    for (int i = 0; i < d->n_laws; i++) if (d->law_type[i] == MEL_LAW_DAMPED_MOHR_COULOMB) D.any_damped = 1;
    // bodies
    h->b_type.assign(d->body_type, d->body_type + nb);
    h->b_status.assign(d->body_status, d->body_status + nb);
    h->b_node0.assign(d->body_node_ptr, d->body_node_ptr + nb + 1);
    h->b_mat.assign(d->body_material, d->body_material + nb);
    D.b_type = dupload(h, d->body_type, nb);
    D.b_mat = dupload(h, d->body_material, nb);
    D.b_per = dupload(h, d->body_periodic, nb);
    D.b_status = dupload(h, d->body_status, nb);
    D.b_damage = dalloc<double>(h, nb);
    MEL_CUDA_OK(cudaMemset(D.b_damage, 0, sizeof(double) * (size_t)nb));
    // DEACTIVATION entries that Update_status compares (Code/Proximity.h:550-1007), checked against
    // the model: the reference indexes its arrays with them unchecked
    if (d->n_deactivated > 0) {
        if (!d->deactivated) { mel_set_error("n_deactivated > 0 without entries"); return MEL_ERR_INVALID; }
        auto nodes_of = [&](int b) { return d->body_node_ptr[b + 1] - d->body_node_ptr[b]; };
        std::vector<double> keep;
        for (int i = 0; i < d->n_deactivated; i++) {
            const double* e = d->deactivated + (size_t)MEL_DEACT_NF * i;
            const int type = (int)e[0];
            if (type == 8) {                                        // Damage: {8, body, mode, threshold}
                const int body = (int)e[1];
                if (body < 0 || body >= nb) { mel_set_error("DEACTIVATION entry %d: body out of range", i); return MEL_ERR_INVALID; }
                keep.insert(keep.end(), e, e + MEL_DEACT_NF);
                continue;
            }
            if (type < 0 || type > 4) continue;                    // Update_status has no branch for it
            const int body = (int)(type <= 3 ? e[2] : e[3]), node = (int)(type <= 3 ? e[3] : e[4]);
            if (body < 0 || body >= nb || node >= nodes_of(body)) { mel_set_error("DEACTIVATION entry %d: body or node out of range", i); return MEL_ERR_INVALID; }
            if (type == 4) {
                const int fk = (int)e[2];
                if (fk < 0 || fk > 7) { mel_set_error("DEACTIVATION entry %d: force kind %d", i, fk); return MEL_ERR_INVALID; }
                if (node < 0 && (fk >= nb || (d->body_type[fk] == MEL_BODY_DEFORMABLE && nodes_of(fk) > nodes_of(body)))) {
                    mel_set_error("DEACTIVATION entry %d: the reference reads the type and node count of body number <force kind> "
                                  "(Code/Proximity.h:866-882), which this model does not allow", i);
                    return MEL_ERR_INVALID;
                }
                if (node >= 0 || d->body_type[fk] == MEL_BODY_DEFORMABLE) h->deact_forces = true;
            }
            keep.insert(keep.end(), e, e + MEL_DEACT_NF);
        }
        if (!keep.empty()) {
            h->d_deact = dupload(h, keep);
            h->n_deact = (int)(keep.size() / MEL_DEACT_NF);
            if (h->deact_forces) D.record_forces = 1;
        }
    }
    D.b_node0 = dupload(h, d->body_node_ptr, nb + 1);
    D.b_bd0 = dupload(h, d->body_border_ptr, nb + 1);
    D.b_dist = dupload(h, d->body_dist, 3 * (size_t)nb);
    std::vector<int> has_bc(nb, 0);
    for (int g = 0; g < nbd; g++)
        if (d->border_bc_type[2 * g] != MEL_BC_NONE || d->border_bc_type[2 * g + 1] != MEL_BC_NONE) has_bc[d->border_body[g]] = 1;
    D.b_has_bc = dupload(h, has_bc);
    // CTA order of the body kernel: rigid bodies, deformable bodies, then the deformable bodies above
    // MEL_MAX_BODY_NODES nodes, which run in a launch of their own (body_kernel_wide)
    std::vector<int> order;
    auto is_wide = [&](int b) { return d->body_type[b] != MEL_BODY_RIGID && d->body_node_ptr[b + 1] - d->body_node_ptr[b] > MEL_MAX_BODY_NODES; };
    for (int b = 0; b < nb; b++) if (d->body_type[b] == MEL_BODY_RIGID) order.push_back(b);
    for (int b = 0; b < nb; b++) if (d->body_type[b] != MEL_BODY_RIGID && !is_wide(b)) order.push_back(b);
    h->nwide = 0;
    for (int b = 0; b < nb; b++) if (is_wide(b)) { order.push_back(b); h->nwide++; }
    D.b_order = dupload(h, order);
    h->nblocks_body = nb - h->nwide;
    // rigid state: file masses first (the first Update_proximity precedes Update_material,
    // Code/main.cpp:112-123); Update_material masses kept for later
    h->rg_file.assign(d->rigid, d->rigid + (size_t)nb * MEL_RIGID_NF);
    h->rg_mat = h->rg_file;
    for (int b = 0; b < nb; b++) {
        double* rg = &h->rg_mat[(size_t)b * MEL_RIGID_NF];
        const double Rho = d->material_params[MEL_MAT_NPARAM * d->body_material[b]];
        int n0 = d->body_node_ptr[b];
        if (d->body_type[b] == MEL_BODY_RIGID) {   // Body::Update_material, rigid branch (Code/Body.h:2867-2905)
            double mass = 0., inertia = 0.;
            for (int c = d->body_cell_ptr[b]; c < d->body_cell_ptr[b + 1]; c++) {
                int a0 = d->cells[3 * c], a1 = d->cells[3 * c + 1], a2 = d->cells[3 * c + 2];
                const double* X = d->node_x0;
                double x0 = X[2 * (n0 + a0)], y0 = X[2 * (n0 + a0) + 1], x1 = X[2 * (n0 + a1)], y1 = X[2 * (n0 + a1) + 1];
                double x2 = X[2 * (n0 + a2)], y2 = X[2 * (n0 + a2) + 1];
                double xc = (x0 + x1 + x2) / 3., yc = (y0 + y1 + y2) / 3.;
                double surf = tri_surface(x0, y0, x1, y1, x2, y2);
                mass += surf;
                inertia += surf * ((xc - rg[MEL_RG_X0]) * (xc - rg[MEL_RG_X0]) + (yc - rg[MEL_RG_Y0]) * (yc - rg[MEL_RG_Y0]));
                inertia += tri_inertia(x0, y0, x1, y1, x2, y2, xc, yc);
            }
            mass *= Rho; inertia *= Rho;
            rg[MEL_RG_MASS] = mass; rg[MEL_RG_INERTIA] = inertia;
            rg[MEL_RG_INV_MASS] = 1. / mass; rg[MEL_RG_INV_INERTIA] = 1. / inertia;
        }
    }
    // rigid bodies start from their centre + displacement (Load_dynamic -> Update_current_positions)
    for (int b = 0; b < nb; b++) {
        if (d->body_type[b] != MEL_BODY_RIGID) continue;
        for (double* rg : { &h->rg_file[(size_t)b * MEL_RIGID_NF], &h->rg_mat[(size_t)b * MEL_RIGID_NF] }) {
            rg[MEL_RG_XC] = rg[MEL_RG_X0] + rg[MEL_RG_XD];
            rg[MEL_RG_YC] = rg[MEL_RG_Y0] + rg[MEL_RG_YD];
            rg[MEL_RG_RC] = rg[MEL_RG_R0] + rg[MEL_RG_RD];
        }
    }
    D.rg = dupload(h, h->rg_file);
    D.rf = dalloc<double>(h, 15 * (size_t)nb);
    D.rtot = dalloc<double>(h, 3 * (size_t)nb);
    D.drv = dalloc<double>(h, 8 * (size_t)nb);
    D.works = dalloc<double>(h, 7 * (size_t)nb);
    // nodes
    std::vector<double> mass(d->node_mass, d->node_mass + 2 * (size_t)nn), minv(d->node_inv_mass, d->node_inv_mass + 2 * (size_t)nn);
    if (d->flags[4] == 1) {   // Body::Update_material, consistent row-sum masses (Code/Body.h:2755-2783)
        for (int b = 0; b < nb; b++) {
            if (d->body_type[b] != MEL_BODY_DEFORMABLE) continue;
            const double Rho = d->material_params[MEL_MAT_NPARAM * d->body_material[b]];
            int n0 = d->body_node_ptr[b];
            for (int i = n0; i < d->body_node_ptr[b + 1]; i++) { mass[2 * i] = 0.; mass[2 * i + 1] = 0.; }
            for (int g = d->body_gp_ptr[b]; g < d->body_gp_ptr[b + 1]; g++)
                for (int j = d->gp_sup_ptr[g]; j < d->gp_sup_ptr[g + 1]; j++)
                    for (int k = d->gp_sup_ptr[g]; k < d->gp_sup_ptr[g + 1]; k++) {
                        double dm = d->gp_weight[g] * d->gp_jacobian[g] * d->gp_N[j] * d->gp_N[k];
                        mass[2 * (n0 + d->gp_sup_idx[j])] += dm;
                        mass[2 * (n0 + d->gp_sup_idx[j]) + 1] += dm;
                    }
            double bm = 0.;
            for (int i = n0; i < d->body_node_ptr[b + 1]; i++) {
                mass[2 * i] *= Rho; mass[2 * i + 1] *= Rho;
                minv[2 * i] = 1. / mass[2 * i]; minv[2 * i + 1] = 1. / mass[2 * i + 1];
                bm += sqrt(mass[2 * i] * mass[2 * i] + mass[2 * i + 1] * mass[2 * i + 1]);
            }
            h->rg_mat[(size_t)b * MEL_RIGID_NF + MEL_RG_MASS] = bm;
            h->rg_mat[(size_t)b * MEL_RIGID_NF + MEL_RG_INV_MASS] = 1 / bm;
        }
    }
    // MATRICES entries, with the stiffness and damping updates of Body::Update_material applied
    // (UPDATE_STIFFNESS_MATRIX, UPDATE_DAMPING_MATRIX; the damping takes the masses above)
    std::vector<double> mk, mc;
    if (d->n_matrix > 0) {
        mk.assign(d->matrix_stiffness, d->matrix_stiffness + d->n_matrix);
        mc.assign(d->matrix_damping, d->matrix_damping + d->n_matrix);
        mel_status st = mel_update_matrices(d, mass.data(), mk.data(), mc.data());
        if (st != MEL_OK) return st;
    }
    h->X0.assign(d->node_x0, d->node_x0 + 2 * (size_t)nn);
    D.X0 = (const double2*)dupload(h, d->node_x0, 2 * (size_t)nn);
    D.mass = (const double2*)dupload(h, mass);
    D.minv = (const double2*)dupload(h, minv);
    D.x = (double2*)dalloc<double>(h, 2 * (size_t)nn);
    D.u = (double2*)dalloc<double>(h, 2 * (size_t)nn);
    D.v = (double2*)dalloc<double>(h, 2 * (size_t)nn);
    D.a = (double2*)dalloc<double>(h, 2 * (size_t)nn);
    D.up = (double2*)dalloc<double>(h, 2 * (size_t)nn);
    D.vp = (double2*)dalloc<double>(h, 2 * (size_t)nn);
    D.ap = (double2*)dalloc<double>(h, 2 * (size_t)nn);
    // damping matrices (Body::Update_damping_forces, Code/Body.h:1057-1154): every entry (dof0, dof1,
    // c) of a deformable body gives the terms the reference's branches add, in their order; bucketed
    // by receiving degree of freedom with the entries' order kept, so each one adds its terms in the
    // reference's sequence
    if (d->n_matrix > 0) {
        std::vector<int> cnt(2 * (size_t)nn + 1, 0);
        auto terms = [&](auto&& emit) {
            for (int b = 0; b < nb; b++) {
                if (d->body_type[b] != MEL_BODY_DEFORMABLE) continue;
                const int n0 = d->body_node_ptr[b];
                for (int i = d->body_matrix_ptr[b]; i < d->body_matrix_ptr[b + 1]; i++) {
                    const int dof0 = d->matrix_dofs[2 * i], dof1 = d->matrix_dofs[2 * i + 1];
                    const int a = 2 * (n0 + dof0 / 2), c = 2 * (n0 + dof1 / 2);
                    const int dir0 = dof0 % 2, dir1 = dof1 % 2;
                    const double cf = mc[i];
                    emit(a + dir0, c + dir1, cf);                               // node0 receives from node1
                    if (dir0 != dir1 || dof0 != dof1) emit(c + dir1, a + dir0, cf); // and node1 from node0
                }
            }
        };
        terms([&](int t, int, double) { cnt[t + 1]++; });
        for (size_t k = 1; k < cnt.size(); k++) cnt[k] += cnt[k - 1];
        if (cnt.back() > 0) {
            std::vector<int> pos(cnt.begin(), cnt.end() - 1), src(cnt.back());
            std::vector<double> cf(cnt.back());
            terms([&](int t, int s_, double c_) { src[pos[t]] = s_; cf[pos[t]] = c_; pos[t]++; });
            D.dmp_ptr = dupload(h, cnt);
            D.dmp_src = dupload(h, src);
            D.dmp_c = dupload(h, cf);
            D.fdamp = (double2*)dalloc<double>(h, 2 * (size_t)nn);
        }
    }
    // ALID layers (Body::Update_alid_forces, Code/Body.h:1163-1296): the bodies whose x or y history
    // is non-empty; per receiving degree of freedom, the terms the reference's entry loop adds when
    // the receiving direction has a history, with d = k / (1/alpha0 + 1/alpha1) evaluated here in the
    // reference's arithmetic
    D.n_alid = 0;
    if (d->body_alid_ptr && d->alid_time && d->alid_value && d->node_alid) {
        const int* hp = d->body_alid_ptr;
        std::vector<int> bl;
        for (int b = 0; b < nb; b++)
            if (d->body_type[b] == MEL_BODY_DEFORMABLE && hp[2 * b + 2] > hp[2 * b]) bl.push_back(b);
        if (!bl.empty()) {
            for (int k = 0; k < 2 * nb; k++)
                if (hp[k + 1] < hp[k]) { mel_set_error("body_alid_ptr must not decrease"); return MEL_ERR_INVALID; }
            const double* ab = d->node_alid;
            std::vector<int> cnt(2 * (size_t)nn + 1, 0);
            auto terms = [&](auto&& emit) {
                for (int b : bl) {
                    if (!d->body_matrix_ptr) break;
                    const int n0 = d->body_node_ptr[b];
                    const bool fl[2] = { hp[2 * b + 1] > hp[2 * b], hp[2 * b + 2] > hp[2 * b + 1] };
                    for (int i = d->body_matrix_ptr[b]; i < d->body_matrix_ptr[b + 1]; i++) {
                        const int dof0 = d->matrix_dofs[2 * i], dof1 = d->matrix_dofs[2 * i + 1];
                        const int a = n0 + dof0 / 2, c = n0 + dof1 / 2;
                        const int dir0 = dof0 % 2, dir1 = dof1 % 2;
                        const double cf = mk[i] / (1. / ab[2 * a] + 1. / ab[2 * c]);
                        if (fl[dir0]) emit(2 * a + dir0, 2 * c + dir1, cf);
                        if ((dir0 != dir1 || dof0 != dof1) && fl[dir1]) emit(2 * c + dir1, 2 * a + dir0, cf);
                    }
                }
            };
            terms([&](int t, int, double) { cnt[t + 1]++; });
            for (size_t k = 1; k < cnt.size(); k++) cnt[k] += cnt[k - 1];
            std::vector<int> pos(cnt.begin(), cnt.end() - 1), src(std::max(cnt.back(), 1), 0);
            std::vector<double> cf(std::max(cnt.back(), 1), 0.);
            terms([&](int t, int s_, double c_) { src[pos[t]] = s_; cf[pos[t]] = c_; pos[t]++; });
            std::vector<double> beta(nn);
            for (int i = 0; i < nn; i++) beta[i] = ab[2 * i + 1];
            const int nh = hp[2 * nb];
            D.n_alid = (int)bl.size();
            D.alid_b = dupload(h, bl);
            D.alid_hptr = dupload(h, std::vector<int>(hp, hp + 2 * nb + 1));
            D.alid_ht = dupload(h, std::vector<double>(d->alid_time, d->alid_time + nh));     // nh >= 1: a body has history
            D.alid_hv = dupload(h, std::vector<double>(d->alid_value, d->alid_value + nh));
            D.alid_beta = dupload(h, beta);
            D.al_ptr = dupload(h, cnt);
            D.al_src = dupload(h, src);
            D.al_c = dupload(h, cf);
            D.falid = (double2*)dalloc<double>(h, 2 * (size_t)nn);
            MEL_CUDA_OK(cudaMemset(D.falid, 0, sizeof(double2) * (size_t)nn));
        }
    }
    // Solver_step state: temporaries, errors, mass-scaling factors (1), estimators (Code/IO.h:1620,1819)
    D.solver = d->solver;
    for (int k = 0; k < 8; k++) D.sp[k] = d->solver_params[k];
    D.upt = (double2*)dalloc<double>(h, 2 * (size_t)nn);
    D.ut = (double2*)dalloc<double>(h, 2 * (size_t)nn);
    D.errv = (double2*)dalloc<double>(h, 2 * (size_t)nn);
    {
        std::vector<double> ones(2 * (size_t)nn, 1.), ide(nn, 0.), bones(nb, 1.);
        for (int b = 0; b < nb; b++)
            for (int i = d->body_node_ptr[b]; i < d->body_node_ptr[b + 1]; i++) {
                if (d->body_type[b] == MEL_BODY_DEFORMABLE) {
                    const int ns = d->node_sup_ptr[i + 1] - d->node_sup_ptr[i];
                    ide[i] = ns ? 1. / (d->node_domain[i] * sqrt(3.1415927 / 4. / ns)) : 0.;
                } else ide[i] = 1. / d->body_dist[3 * b];
            }
        D.fms = (double2*)dupload(h, ones);
        D.ide = dupload(h, ide);
        D.bfms = dupload(h, bones);
    }
    D.terr = dalloc<double>(h, nb);
    D.merr = dalloc<double>(h, nb);
    D.bmms = dalloc<double>(h, nb);
    D.bdfms = dalloc<double>(h, nb);
    D.rg_tmp = dalloc<double>(h, 6 * (size_t)nb);
    h->nse = d->node_sup_ptr[nn];
    std::vector<uint16_t> sidx(h->nse);
    for (int b = 0; b < nb; b++)
        for (int i = d->body_node_ptr[b]; i < d->body_node_ptr[b + 1]; i++)
            for (int j = d->node_sup_ptr[i]; j < d->node_sup_ptr[i + 1]; j++) {
                int v = d->node_sup_idx[j];
                if (v < 0 || v >= d->body_node_ptr[b + 1] - d->body_node_ptr[b]) { mel_set_error("node support index out of range"); return MEL_ERR_INVALID; }
                sidx[j] = (uint16_t)v;
            }
    D.sup_ptr = dupload(h, d->node_sup_ptr, nn + 1);
    D.sup_idx = dupload(h, sidx);
    D.sup_N = dupload(h, d->node_sup_N, h->nse);
    {
        // kinematics layout (mel_dev::ks_*): a warp's 32 slots read row k of their supports as 32
        // consecutive entries; each node's supports keep their order
        std::vector<int> ks0(nb + 1, 0), kgb;
        std::vector<unsigned> rec;
        std::vector<uint16_t> kidx;
        std::vector<double> kN;
        std::vector<int> order;
        for (int b = 0; b < nb; b++) {
            ks0[b] = (int)rec.size();
            if (d->body_type[b] != MEL_BODY_DEFORMABLE) continue;
            const int b0 = d->body_node_ptr[b], nbn = d->body_node_ptr[b + 1] - b0;
            order.resize(nbn);
            std::iota(order.begin(), order.end(), 0);
            auto cnt = [&](int i) { return d->node_sup_ptr[b0 + i + 1] - d->node_sup_ptr[b0 + i]; };
            std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return cnt(x) > cnt(y); });
            for (int s0 = 0; s0 < nbn; s0 += 32) {
                const int m = std::min(32, nbn - s0);
                const int K = cnt(order[s0]);
                const size_t base = kidx.size();
                kgb.push_back((int)base);
                kidx.resize(base + 32 * (size_t)K, 0);
                kN.resize(base + 32 * (size_t)K, 0.);
                for (int l = 0; l < m; l++) {
                    const int i = order[s0 + l];
                    if (cnt(i) > 0xffff) { mel_set_error("node %d has %d supports", b0 + i, cnt(i)); return MEL_ERR_UNSUPPORTED; }
                    rec.push_back((unsigned)i | ((unsigned)cnt(i) << 16));
                    for (int k = 0, j = d->node_sup_ptr[b0 + i]; k < cnt(i); k++, j++) {
                        kidx[base + 32 * (size_t)k + l] = sidx[j];
                        kN[base + 32 * (size_t)k + l] = d->node_sup_N[j];
                    }
                }
                for (int l = m; l < 32; l++) rec.push_back(0u);
            }
            if (kidx.size() > (size_t)INT32_MAX) { mel_set_error("node supports above 2^31 entries"); return MEL_ERR_UNSUPPORTED; }
        }
        ks0[nb] = (int)rec.size();
        if (rec.empty()) { rec.push_back(0u); kgb.push_back(0); kidx.push_back(0); kN.push_back(0.); }
        D.b_ks0 = dupload(h, ks0);
        D.ks_rec = dupload(h, rec);
        D.kg_base = dupload(h, kgb);
        D.ks_idx = dupload(h, kidx);
        D.ks_N = dupload(h, kN);
    }
    D.o_fint = (double2*)dalloc<double>(h, 2 * (size_t)nn);
    D.o_fcon = (double2*)dalloc<double>(h, 2 * (size_t)nn);
    D.o_fneu = (double2*)dalloc<double>(h, 2 * (size_t)nn);
    D.o_fdir = (double2*)dalloc<double>(h, 2 * (size_t)nn);
    D.o_ftot = (double2*)dalloc<double>(h, 2 * (size_t)nn);
    // borders
    D.bd_body = dupload(h, d->border_body, nbd);
    D.bd_per = dupload(h, d->border_periodicity, nbd);
    D.bd_bef = dupload(h, d->border_before, nbd);
    D.bd_aft = dupload(h, d->border_after, nbd);
    D.bd_e0 = dupload(h, d->border_node_ptr, nbd + 1);
    D.bd_bc = dupload(h, d->border_bc_type, 2 * (size_t)nbd);
    D.bd_bcp = dupload(h, d->border_bc_param, 4 * (size_t)nbd);
    D.bd_h0 = dupload(h, d->border_hist_ptr, 2 * (size_t)nbd + 1);
    int nh = d->border_hist_ptr[2 * nbd];
    D.ht = dupload(h, d->hist_time, nh);
    D.hv = dupload(h, d->hist_value, nh);
    D.e_node = dupload(h, d->border_nodes, ne);
    std::vector<int> sn(4 * (size_t)ne, 0), ss(4 * (size_t)ne, 0);
    std::vector<double> len0(ne, 0.);
    for (int b = 0; b < nb; b++) initialize_segments(d, b, sn, ss, len0);
    D.e_sn = dupload(h, sn);
    D.e_ss = dupload(h, ss);
    D.e_len0 = dupload(h, len0);
    std::vector<double> len(len0);
    D.e_len = dupload(h, len);
    D.e_bcp = dalloc<double2>(h, (size_t)ne + 1);
    D.cp_cnt = dalloc<int>(h, (size_t)ne + 1);
    D.cp_item = dalloc<int>(h, (size_t)(ne > 0 ? ne : 1) * MEL_PRESSURE_CAP);
    D.cpx = dalloc<double>(h, (size_t)ne + 1);
    D.cpy = dalloc<double>(h, (size_t)ne + 1);
    {
        std::vector<int> blk0(nbd + 1, 0), blk_border;
        for (int g = 0; g < nbd; g++) {
            int nseg = d->border_node_ptr[g + 1] - d->border_node_ptr[g] - 1;
            int nbk = (nseg + MEL_SEGB - 1) / MEL_SEGB;
            blk0[g + 1] = blk0[g] + nbk;
            for (int k = 0; k < nbk; k++) blk_border.push_back(g);
        }
        D.nblk = blk0[nbd];
        D.bd_blk0 = dupload(h, blk0);
        D.blk_border = dupload(h, blk_border);
        D.seg_blk = (double4*)dalloc<double>(h, 4 * (size_t)(D.nblk + 1));
        std::vector<int> sblk0(nbd + 1, 0), sblk_border;
        for (int g = 0; g < nbd; g++) {
            int nsb = (blk0[g + 1] - blk0[g] + MEL_SEGB2 - 1) / MEL_SEGB2;
            sblk0[g + 1] = sblk0[g] + nsb;
            for (int k = 0; k < nsb; k++) sblk_border.push_back(g);
        }
        D.nsblk = sblk0[nbd];
        D.bd_sblk0 = dupload(h, sblk0);
        D.sblk_border = dupload(h, sblk_border);
        D.seg_sblk = (double4*)dalloc<double>(h, 4 * (size_t)(D.nsblk + 1));
    }
    h->H.b_type = h->b_type;
    h->H.b_per.assign(d->body_periodic, d->body_periodic + nb);
    h->H.b_bd0.assign(d->body_border_ptr, d->body_border_ptr + nb + 1);
    h->H.bd_e0.assign(d->border_node_ptr, d->border_node_ptr + nbd + 1);
    // Gauss points: chunk images of <= gpcap points (one point thread each) and <= ecap support
    // entries.  The entry cap is the largest that lets two body CTAs, each with its ring of
    // MEL_STAGES images, share an SM; a body too large for that runs one CTA per SM.
    // Bodies above MEL_MAX_BODY_NODES nodes keep their node arrays in global memory (gscr), so
    // shared memory is sized by the others (max_def_nodes); max_all_nodes bounds the touched nodes
    // of a chunk.
    int max_def_nodes = 1, max_all_nodes = 1;
    bool any_wide = false;
    for (int b = 0; b < nb; b++)
        if (d->body_type[b] == MEL_BODY_DEFORMABLE) {
            const int nnb = d->body_node_ptr[b + 1] - d->body_node_ptr[b];
            max_all_nodes = std::max(max_all_nodes, nnb);
            if (nnb > MEL_MAX_BODY_NODES) any_wide = true;
            else max_def_nodes = std::max(max_def_nodes, nnb);
        }
    if (any_wide) {
        // per wide body: s_f, s_fc (16 B per node), s_upf (8 B, mixed), then the post-loop arrays
        // s_fn, s_fd, s_vp, s_ap (16 B), six work terms (48 B) and the temporary parameters (16 B)
        std::vector<long long> off(nb, -1);
        long long tot = 0;
        for (int b = 0; b < nb; b++) {
            const int nnb = d->body_node_ptr[b + 1] - d->body_node_ptr[b];
            if (d->body_type[b] != MEL_BODY_DEFORMABLE || nnb <= MEL_MAX_BODY_NODES) continue;
            off[b] = tot;
            tot += ((long long)mel_wide_bytes(nnb) + 255) & ~255LL;
        }
        D.b_gscr = dupload(h, off);
        D.gscr = reinterpret_cast<char*>(dalloc<double>(h, (size_t)(tot / 8) + 32));
    }
    mel_chunk_set CS;
    long long pipe_min = 0;
    int smem_sm = 0, smem_blk = 0, smem_res = 0;
    cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, h->device);
    cudaDeviceGetAttribute(&smem_blk, cudaDevAttrMaxSharedMemoryPerBlockOptin, h->device);
    cudaDeviceGetAttribute(&smem_res, cudaDevAttrReservedSharedMemoryPerBlock, h->device);
    const size_t two_per_sm = (size_t)(smem_sm / 2 - smem_res);
    {
        const bool mixed = h->precision == MEL_PREC_MIXED;
        // which mixed bodies run the three-stage pipeline: those with at least pipe_min support
        // entries (MELGPU_PIPE_MIN_ENTRIES overrides the default); the others run the two-buffer loop
        if (mixed) {
            pipe_min = MEL_PIPE_MIN_ENTRIES;
            if (const char* e = getenv("MELGPU_PIPE_MIN_ENTRIES")) pipe_min = atoll(e);
        }
        bool any_pipe = false, any_loop = false;
        for (int b = 0; b < nb; b++)
            if (d->body_type[b] == MEL_BODY_DEFORMABLE) {
                if (mixed && mel_body_entries(d, b) >= pipe_min) any_pipe = true; else any_loop = true;
            }
        const int stages = any_pipe ? MEL_STAGES(1) : 2;
        // FP32 images hold 12 bytes per entry instead of 20; pipeline bodies have fewer point threads
        const int gpcap = any_loop ? MEL_CHUNK_GP_FP64 : MEL_CHUNK_GP_MX;
        const int caps_fp64[] = { MEL_CHUNK_E_MAX, 1792, 1536, 1408, 1344, 1280, 1216, 1152, 1024, 768, 512, 256 };
        const int caps_mixed[] = { MEL_CHUNK_E_MAX, 1920, 1792, 1664, 1536, 1408, 1280, 1024, 768, 512, 256 };
        std::vector<int> caps = mixed ? std::vector<int>(std::begin(caps_mixed), std::end(caps_mixed))
                                      : std::vector<int>(std::begin(caps_fp64), std::end(caps_fp64));
        // the cap is chosen from an upper bound of the image size (a chunk holds at most ecap
        // entries, gpcap points, min(ecap, nodes) touched nodes and one row per support
        // of each group's largest point), so the images are built once
        // Pull rows: the first pull group has at most (the most points any node supports) rows,
        // and each later group at most its predecessor's smallest count, so all later groups
        // together at most ecap / 32.
        int max_ns = 1, max_use = 1;
        std::vector<int> use;
        for (int b = 0; b < nb; b++)
            if (d->body_type[b] == MEL_BODY_DEFORMABLE) {
                use.assign(d->body_node_ptr[b + 1] - d->body_node_ptr[b], 0);
                for (int g = d->body_gp_ptr[b]; g < d->body_gp_ptr[b + 1]; g++) {
                    max_ns = std::max(max_ns, d->gp_sup_ptr[g + 1] - d->gp_sup_ptr[g]);
                    for (int j = d->gp_sup_ptr[g]; j < d->gp_sup_ptr[g + 1]; j++) {
                        const int v = d->gp_sup_idx[j];
                        if (v >= 0 && v < (int)use.size()) max_use = std::max(max_use, ++use[v]);
                    }
                }
            }
        auto bound = [&](int ecap) {
            const int ne = std::min(ecap, gpcap * max_ns);
            const int groups = (gpcap + 31) / 32;
            const int pull_rows = std::min(max_use, gpcap) + ne / 32;
            // pull records: touched-node slots, or (mixed two-buffer loop) the segmented list
            // pull records: touched-node slots, or (mixed two-buffer loop) the warp bounds and at most
            // one piece per touched node plus one per MEL_PIECE entries
            int tn_words = std::max(std::min(ne, max_all_nodes), mixed ? 5 + std::min(ne, max_all_nodes) + ne / MEL_PIECE : 0);
            if (any_wide && !mixed) tn_words += (tn_words + 1) / 2 + 4;     // the 16-bit node section of wide bodies
            return mel_chunk_sections(gpcap, ne, tn_words, std::min(1023, groups * max_ns) + pull_rows, mixed ? 8 : 16).bytes;
        };
        int chosen = -1;
        // a cap from the tuning table (MELGPU_TUNE_FILE, written by melody2d_b200.autotune), or forced
        // by MELGPU_CHUNK_CAP (the tuner's own runs), is taken when it fits the shared memory
        const int tuned = tuned_chunk_cap(h->precision, max_def_nodes);
        if (tuned > 0 && mel_body_smem_bytes(max_def_nodes, bound(tuned), mixed, stages) <= (size_t)smem_blk) chosen = tuned;
        if (chosen < 0)
            for (int ecap : caps)
                if (mel_body_smem_bytes(max_def_nodes, bound(ecap), mixed, stages) <= two_per_sm) { chosen = ecap; break; }
        if (chosen < 0)     // one CTA per SM: largest cap that fits
            for (int ecap : caps)
                if (mel_body_smem_bytes(max_def_nodes, bound(ecap), mixed, stages) <= (size_t)smem_blk) { chosen = ecap; break; }
        if (chosen < 0) {
            mel_set_error("deformable body of %d nodes does not fit the body kernel's shared memory", max_def_nodes);
            return MEL_ERR_UNSUPPORTED;
        }
        mel_status rc = mel_build_chunks(d, chosen, CS, mixed, pipe_min);
        if (rc) return rc;
        h->chunk_cap = chosen;
    }
    h->nge = (int)CS.n_entries;
    h->n_pad = CS.n_pad;
    D.nchunk = (int)CS.chunks.size();
    D.chunk = dupload(h, CS.chunks);
    D.b_chunk0 = dupload(h, CS.b_chunk0);
    D.img = reinterpret_cast<const char*>(dupload(h, CS.img));
    D.img_cap = CS.img_max;
    if (h->precision == MEL_PREC_MIXED) D.b_pipe = dupload(h, CS.b_pipe);
    h->body_stages = 2;
    for (int v : CS.b_pipe) if (v) h->body_stages = MEL_STAGES(1);
    h->img_bytes = (double)CS.img.size();
    // contacts and proximity buffers
    D.err = dalloc<unsigned>(h, MEL_E_NWORDS);
    D.ncont = 0;
    mel_prox_state& P = h->P;
    P.nbr_cap = MEL_NBR_CAP_DEFAULT;
    if (cudaMalloc(&P.nbr, sizeof(int) * 3 * (size_t)P.nbr_cap * nb) != cudaSuccess) return MEL_ERR_OOM;
    P.nbn = dalloc<int>(h, nb);
    P.aabb = dalloc<double>(h, 4 * (size_t)nbd);
    P.shmin = dalloc<int>(h, nbd);
    P.shmax = dalloc<int>(h, nbd);
    {
        // cell-list broad phase for models of at least MELGPU_CELL_MIN_BODIES bodies (default 64;
        // smaller ones take the all-pairs pass): cells 1.5 x the largest initial border box of a
        // deformable body (with its detection distance), so a grain's box covers at most 2 x 2 cells
        int min_bodies = 64;
        if (const char* e = getenv("MELGPU_CELL_MIN_BODIES")) min_bodies = atoi(e);
        double ext = 0., ext_all = 0.;
        for (int b = 0; b < nb; b++) {
            const int n0 = d->body_node_ptr[b];
            const double det = d->body_dist[3 * b + 1];
            for (int g = d->body_border_ptr[b]; g < d->body_border_ptr[b + 1]; g++) {
                double x0 = 1e300, x1 = -1e300, y0 = 1e300, y1 = -1e300;
                for (int k = d->border_node_ptr[g]; k < d->border_node_ptr[g + 1]; k++) {
                    const int i = n0 + d->border_nodes[k];
                    x0 = std::min(x0, d->node_x0[2 * i]); x1 = std::max(x1, d->node_x0[2 * i]);
                    y0 = std::min(y0, d->node_x0[2 * i + 1]); y1 = std::max(y1, d->node_x0[2 * i + 1]);
                }
                const double e = std::max(x1 - x0, y1 - y0) + 2. * det;
                if (std::isfinite(e)) {
                    ext_all = std::max(ext_all, e);
                    if (d->body_type[b] == MEL_BODY_DEFORMABLE) ext = std::max(ext, e);
                }
            }
        }
        if (ext <= 0.) ext = ext_all;
        const double period = d->period[1] - d->period[0];
        if (nb >= min_bodies && ext > 0. && std::isfinite(period) && period > 0.) {
            P.cl_on = 1;
            P.cl_h = 1.5 * ext;
            P.cl_ncx = (int)std::max(1., std::min(1e6, std::floor(period / P.cl_h)));
            P.cl_hx = period / P.cl_ncx;
            P.cl_T = 64;
            while (P.cl_T < 2 * nbd) P.cl_T *= 2;
            P.cl_cnt = dalloc<int>(h, P.cl_T + 1);
            P.cl_cur = dalloc<int>(h, P.cl_T + 1);
            P.cl_start = dalloc<int>(h, P.cl_T + 1);
            P.cl_idx = dalloc<int>(h, nbd);
            P.cl_w = reinterpret_cast<unsigned long long*>(dalloc<double>(h, 2));
        }
    }
    P.b_inc0 = dalloc<int>(h, nb + 1);
    P.tcnt = dalloc<int>(h, nb + 1);
    P.btask0 = dalloc<int>(h, nb + 2);
    P.scnt = dalloc<int>(h, nb + 1);
    P.bslot0 = dalloc<int>(h, nb + 2);
    P.b_cont0 = dalloc<int>(h, nb + 1);
    P.e_cnt = dalloc<int>(h, ne + 1);
    P.e_ptr = dalloc<int>(h, ne + 2);
    P.e_cur = dalloc<int>(h, ne + 2);
    size_t cb = sizeof(mel_contact) * 1024;
    if (cudaMalloc(&D.cont, cb) != cudaSuccess) return MEL_ERR_OOM;
    P.cont_bytes = cb;
    if (cudaMalloc(&P.cont_w, sizeof(double) * 1024) != cudaSuccess) return MEL_ERR_OOM;
    P.cont_w_bytes = sizeof(double) * 1024;
    D.cont_w = P.cont_w;
    if (cudaMalloc(&P.cont_rt, 6 * sizeof(double) * 1024) != cudaSuccess) return MEL_ERR_OOM;
    P.cont_rt_bytes = 6 * sizeof(double) * 1024;
    D.cont_rt = P.cont_rt;
    D.b_cont0 = P.b_cont0; D.b_inc0 = P.b_inc0;
    if (cudaMalloc(&P.inc_rng, sizeof(int2) * 16) != cudaSuccess) return MEL_ERR_OOM;
    P.inc_rng_bytes = sizeof(int2) * 16;
    D.inc_rng = P.inc_rng;
    h->body_smem = mel_body_smem_bytes(max_def_nodes, CS.img_max, h->precision == MEL_PREC_MIXED, h->body_stages);
    if (mel_body_kernel_configure(h->body_smem) != MEL_OK) return MEL_ERR_CUDA;
    h->d_monitor = dalloc<double>(h, 32);
    h->d_monitor_part = dalloc<double>(h, 5 * 148);
    {
        std::vector<int> rid;
        for (int b = 0; b < nb; b++) if (d->body_type[b] == MEL_BODY_RIGID) rid.push_back(b);
        h->nrigid = (int)rid.size();
        h->d_rigid_ids = dupload(h, rid);
    }
    // algorithmic bytes moved by one launch of each step kernel (exact array sizes):
    // body kernel: the chunk images without their padding entries (entries: dN/dx,dN/dy + 16-bit
    // index + 16-bit pull position; points: c0 + slot record; touched-node records; row tables)
    // and the chunk table; node state read (up,
    // vp, m, 1/m, X0) and written (up, vp, ap, u, v, a, x); node supports (16-bit index + N) and
    // their offsets.  Contact records are left out (a few hundred bytes per body).
    {
        double nd = 0;
        for (int b = 0; b < nb; b++) if (d->body_type[b] == MEL_BODY_DEFORMABLE) nd += d->body_node_ptr[b + 1] - d->body_node_ptr[b];
        h->n_def_nodes = (int)nd;
        double nse_def = 0;
        for (int b = 0; b < nb; b++)
            if (d->body_type[b] == MEL_BODY_DEFORMABLE)
                nse_def += d->node_sup_ptr[d->body_node_ptr[b + 1]] - d->node_sup_ptr[d->body_node_ptr[b]];
        const double entry_bytes = h->precision == MEL_PREC_MIXED ? 12. : 20.;
        h->bytes_body = h->img_bytes - entry_bytes * (double)h->n_pad + (double)CS.chunks.size() * sizeof(mel_chunk) + nd * (5 * 16 + 7 * 16) +
                        nse_def * (2 + 8) + (nd + 1) * 4;
        h->bytes_contact = (double)ne * (4 * 4 + 4 * 4 + 8 + 8);   // refreshed border lengths (contacts added per call)
    }
    if (cudaDeviceSynchronize() != cudaSuccess) { mel_set_cuda_error(cudaGetLastError(), "build", __FILE__, __LINE__); return MEL_ERR_CUDA; }
    return MEL_OK;
}

// ---------------------------------------------------------------------------------------------
// set-up and stepping
// ---------------------------------------------------------------------------------------------
static mel_status check_errors(mel_handle* h)
{
    unsigned w[MEL_E_NWORDS];
    if (cudaMemcpy(w, h->d.err, sizeof w, cudaMemcpyDeviceToHost) != cudaSuccess) { mel_set_cuda_error(cudaGetLastError(), "err", __FILE__, __LINE__); return MEL_ERR_CUDA; }
    if (w[MEL_E_BOUNDS]) { mel_set_error("device index check failed (code %u)", w[MEL_E_BOUNDS]); return MEL_ERR_BOUNDS; }
    if (w[MEL_E_WAIT]) { mel_set_error("a wait of the body kernel's pipeline gave up after %llu ns", h->d.wait_ns); return MEL_ERR_TIMEOUT; }
    if (w[MEL_E_DEACT]) {
        mel_set_error("body %u turned inactive while one of its contact elements carried a force: the reference keeps "
                      "sending that force to the other bodies for the rest of the run (its send list is no longer cleared, "
                      "Code/Solver.h:37-61), which this library does not reproduce", w[MEL_E_DEACT] - 1);
        return MEL_ERR_UNSUPPORTED;
    }
    return MEL_OK;
}

// One proximity update.  With e0/e1 given, they bracket it on the stream (read after the
// caller's final synchronisation, so timing adds no host wait).
static mel_status proximity(mel_handle* h, cudaEvent_t e0 = nullptr, cudaEvent_t e1 = nullptr)
{
    if (e0) cudaEventRecord(e0, h->stream);
    int launches0 = h->P.launches;
    int rc = mel_run_proximity(h->d, h->P, h->H, h->stream);
    h->launches += h->P.launches - launches0;
    if (e1) cudaEventRecord(e1, h->stream);
    if (rc) return (mel_status)rc;      // the pipeline has set the message
    return MEL_OK;
}

static void update_borders_only(mel_handle* h)
{
    mel_dev d = h->d;
    d.ncont = 0;
    mel_launch_contact(d, 1.0, h->stream);
}

static mel_status setup(mel_handle* h)
{
    // Code/main.cpp:104-127: Update_borders, Update_bc, Update_proximity, Initialize_CZM,
    // Update_material, Update_proximity.  Update_bc values are evaluated when used.
    // rigid nodes take their positions from the body state
    std::vector<double> st(12 * (size_t)h->nn, 0.);
    mel_status rc = MEL_OK;
    mel_launch_drivendof(h->d, h->time, h->stream);     // Update_bc(Time): the first half-step of
                                                         // Solver_step moves driven bodies with these
    update_borders_only(h);
    if ((rc = proximity(h))) return rc;
    if (h->flags[3] == 1) {
        // Initialize_CZM (Code/Proximity.h:481-541) runs once: it clears the flag, so the call after
        // the second proximity update does nothing
        mel_launch_czm_init(h->d, h->stream);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) { mel_set_cuda_error(e, "Initialize_CZM launch", __FILE__, __LINE__); return MEL_ERR_CUDA; }
        h->flags[3] = 0;
    }
    cudaMemcpyAsync(h->d.rg, h->rg_mat.data(), sizeof(double) * h->rg_mat.size(), cudaMemcpyHostToDevice, h->stream);
    if ((rc = proximity(h))) return rc;
    if (cudaStreamSynchronize(h->stream) != cudaSuccess) { mel_set_cuda_error(cudaGetLastError(), "setup", __FILE__, __LINE__); return MEL_ERR_CUDA; }
    return check_errors(h);
}

// node positions from node_state (deformable: X0 + u, Code/Node.h:233-237) and rigid body state
// (Code/Body.h:2272-2300), uploaded together
static mel_status upload_state(mel_handle* h, const double* st, const double* rigid)
{
    const int nn = h->nn;
    std::vector<double> u(2 * (size_t)nn), v(2 * (size_t)nn), a(2 * (size_t)nn), up(2 * (size_t)nn), vp(2 * (size_t)nn), ap(2 * (size_t)nn), x(2 * (size_t)nn);
    std::vector<double> rg(rigid ? std::vector<double>(rigid, rigid + (size_t)h->nb * MEL_RIGID_NF) : std::vector<double>());
    if (!rigid) {
        rg.resize((size_t)h->nb * MEL_RIGID_NF);
        cudaMemcpy(rg.data(), h->d.rg, sizeof(double) * rg.size(), cudaMemcpyDeviceToHost);
    }
    if (!st) {
        std::vector<double> tmp(12 * (size_t)nn);
        mel_get_node_state(h, tmp.data());
        return upload_state(h, tmp.data(), rg.data());
    }
    for (int i = 0; i < nn; i++) {
        const double* s = st + 12 * (size_t)i;
        for (int k = 0; k < 2; k++) {
            u[2 * i + k] = s[k]; v[2 * i + k] = s[2 + k]; a[2 * i + k] = s[4 + k];
            up[2 * i + k] = s[6 + k]; vp[2 * i + k] = s[8 + k]; ap[2 * i + k] = s[10 + k];
            x[2 * i + k] = h->X0[2 * i + k] + u[2 * i + k];
        }
    }
    for (int b = 0; b < h->nb; b++) {
        if (h->b_type[b] != MEL_BODY_RIGID) continue;
        double* r = &rg[(size_t)b * MEL_RIGID_NF];
        r[MEL_RG_XC] = r[MEL_RG_X0] + r[MEL_RG_XD];
        r[MEL_RG_YC] = r[MEL_RG_Y0] + r[MEL_RG_YD];
        r[MEL_RG_RC] = r[MEL_RG_R0] + r[MEL_RG_RD];
        double dr = r[MEL_RG_RD] - r[MEL_RG_R0];
        for (int i = h->b_node0[b]; i < h->b_node0[b + 1]; i++) {
            double dx = h->X0[2 * i] - r[MEL_RG_X0], dy = h->X0[2 * i + 1] - r[MEL_RG_Y0];
            x[2 * i] = r[MEL_RG_XC] + dx * mel_cos(dr) - dy * mel_sin(dr);
            x[2 * i + 1] = r[MEL_RG_YC] + dx * mel_sin(dr) + dy * mel_cos(dr);
            double ddx = x[2 * i] - r[MEL_RG_XC], ddy = x[2 * i + 1] - r[MEL_RG_YC];
            v[2 * i] = -ddy * r[MEL_RG_RV] + r[MEL_RG_XV];
            v[2 * i + 1] = ddx * r[MEL_RG_RV] + r[MEL_RG_YV];
        }
    }
    size_t bytes = sizeof(double) * 2 * (size_t)nn;
    MEL_CUDA_OK(cudaMemcpy(h->d.u, u.data(), bytes, cudaMemcpyHostToDevice));
    MEL_CUDA_OK(cudaMemcpy(h->d.v, v.data(), bytes, cudaMemcpyHostToDevice));
    MEL_CUDA_OK(cudaMemcpy(h->d.a, a.data(), bytes, cudaMemcpyHostToDevice));
    MEL_CUDA_OK(cudaMemcpy(h->d.up, up.data(), bytes, cudaMemcpyHostToDevice));
    MEL_CUDA_OK(cudaMemcpy(h->d.vp, vp.data(), bytes, cudaMemcpyHostToDevice));
    MEL_CUDA_OK(cudaMemcpy(h->d.ap, ap.data(), bytes, cudaMemcpyHostToDevice));
    MEL_CUDA_OK(cudaMemcpy(h->d.x, x.data(), bytes, cudaMemcpyHostToDevice));
    MEL_CUDA_OK(cudaMemcpy(h->d.rg, rg.data(), sizeof(double) * rg.size(), cudaMemcpyHostToDevice));
    return MEL_OK;
}

// ---------------------------------------------------------------------------------------------
// Solver_step (Code/Solver.h:98-486): Body::Store / Body::Restore as device copies
// ---------------------------------------------------------------------------------------------
// snapshot: node blob (x, u, v, a, up, vp, ap, upt, ut, fms, errv), works, bdfms, rigid records,
// contact list
static mel_status adaptive_store(mel_handle* h, bool restore)
{
    mel_dev& D = h->d;
    const size_t nn = (size_t)h->nn, nb = (size_t)h->nb;
    double2* nodes[11] = { D.x, D.u, D.v, D.a, D.up, D.vp, D.ap, D.upt, D.ut, D.fms, D.errv };
    if (h->store_bufs.empty()) {
        void* p[3] = { nullptr, nullptr, nullptr };
        if (cudaMalloc(&p[0], sizeof(double2) * 11 * nn) != cudaSuccess ||
            cudaMalloc(&p[1], sizeof(double) * (8 + MEL_RIGID_NF) * nb) != cudaSuccess) {
            for (void* q : p) if (q) cudaFree(q);
            mel_set_error("Solver_step snapshot allocation failed");
            return MEL_ERR_OOM;
        }
        h->store_bufs = { p[0], p[1], nullptr };
        h->store_cont_cap = 0;
    }
    double2* nb_ = static_cast<double2*>(h->store_bufs[0]);
    double* bb = static_cast<double*>(h->store_bufs[1]);
    cudaStream_t s = h->stream;
    const cudaMemcpyKind k = cudaMemcpyDeviceToDevice;
    if (!restore) {
        if ((size_t)D.ncont > h->store_cont_cap) {
            if (h->store_bufs[2]) cudaFree(h->store_bufs[2]);
            h->store_bufs[2] = nullptr;
            const size_t cap = (size_t)D.ncont * 2 + 64;
            if (cudaMalloc(&h->store_bufs[2], sizeof(mel_contact) * cap) != cudaSuccess) {
                h->store_bufs[2] = nullptr; h->store_cont_cap = 0;
                mel_set_error("Solver_step snapshot allocation failed");
                return MEL_ERR_OOM;
            }
            h->store_cont_cap = cap;
        }
        for (int a = 0; a < 11; a++) MEL_CUDA_OK(cudaMemcpyAsync(nb_ + a * nn, nodes[a], sizeof(double2) * nn, k, s));
        MEL_CUDA_OK(cudaMemcpyAsync(bb, D.works, sizeof(double) * 7 * nb, k, s));
        MEL_CUDA_OK(cudaMemcpyAsync(bb + 7 * nb, D.bdfms, sizeof(double) * nb, k, s));
        MEL_CUDA_OK(cudaMemcpyAsync(bb + 8 * nb, D.rg, sizeof(double) * MEL_RIGID_NF * nb, k, s));
        if (D.ncont) MEL_CUDA_OK(cudaMemcpyAsync(h->store_bufs[2], D.cont, sizeof(mel_contact) * D.ncont, k, s));
        h->store_ncont = D.ncont;
    } else {
        for (int a = 0; a < 11; a++) MEL_CUDA_OK(cudaMemcpyAsync(nodes[a], nb_ + a * nn, sizeof(double2) * nn, k, s));
        MEL_CUDA_OK(cudaMemcpyAsync(D.works, bb, sizeof(double) * 7 * nb, k, s));
        MEL_CUDA_OK(cudaMemcpyAsync(D.bdfms, bb + 7 * nb, sizeof(double) * nb, k, s));
        mel_launch_rigid_restore(D, bb + 8 * nb, s);
        MEL_CUDA_OK(cudaGetLastError());
        if (h->store_ncont) MEL_CUDA_OK(cudaMemcpyAsync(D.cont, h->store_bufs[2], sizeof(mel_contact) * h->store_ncont, k, s));
    }
    return MEL_OK;
}

// Deltat's correction law shared by the schemes (Code/Solver.h:349-357)
static void dt_law(mel_handle* h, double c1, double c2)
{
    if (c1 > c2) h->dt = h->dt / pow(c1, h->d.sp[1]);
    else h->dt = h->dt / pow(c2, h->d.sp[1]);
    if (h->dt > h->cup) h->dt = h->cup;
}

// One accepted step of Solver_step: two half-steps with the temporary full step beside the first,
// the error (and mass-scaling) sums, and the scheme's accept / reject rule with its Deltat law;
// a rejected attempt restores the snapshot and retries with the corrected Deltat.  Like the oracle,
// gives up after 1000 attempts (the reference would retry for ever).
static mel_status adaptive_step(mel_handle* h)
{
    if (!h->h_red) {
        if (cudaMallocHost(&h->h_red, 8 * sizeof(double)) != cudaSuccess) { h->h_red = nullptr; mel_set_error("pinned allocation failed"); return MEL_ERR_OOM; }
        h->d_red = dalloc<double>(h, 8);
        if (!h->d_red) { mel_set_error("device allocation failed"); return MEL_ERR_OOM; }
    }
    mel_status rc = adaptive_store(h, false);
    if (rc) return rc;
    const double Target_error = h->d.sp[0], Accepted_ratio = h->d.sp[2], Inv_Target_error = h->d.sp[7];
    int neval = 0;
    bool ok = false;
    double mean_error = 0., max_error = 0., total_mass = 0., max_mass = 0.;
    while (!ok) {
        neval++;
        h->h_red[7] = h->dt;
        MEL_CUDA_OK(cudaMemcpyAsync(h->d.dt, &h->h_red[7], sizeof(double), cudaMemcpyHostToDevice, h->stream));
        mel_dev d = h->d;
        mel_launch_contact(d, 0.5, h->stream);                 // Update_contact_forces(Deltat*0.5)
        mel_launch_damping(d, h->stream);
        mel_launch_alid(d, 0, h->time, 1, h->stream);            // Update_alid_forces(Time)
        d.phase = 1;
        mel_launch_body_adaptive(d, h->time, h->t_bc, h->nblocks_body, h->body_smem, h->stream, h->nwide);
        mel_launch_contact(d, 0.5, h->stream);
        mel_launch_damping(d, h->stream);
        mel_launch_alid(d, 0, h->time + h->dt * 0.5, 1, h->stream);   // Update_alid_forces(Time+Deltat*0.5)
        d.phase = 2;
        mel_launch_body_adaptive(d, h->time, h->time + h->dt * 0.5, h->nblocks_body, h->body_smem, h->stream, h->nwide);
        h->t_bc = h->time + h->dt;                              // Update_bc(Time+Deltat) of the second half
        mel_launch_error_reduce(d, h->d_red, h->stream);
        h->launches += 5 + (h->d.fdamp ? 2 : 0) + (h->d.falid ? 2 : 0) + (h->nwide && h->nblocks_body ? 2 : 0);
        MEL_CUDA_OK(cudaGetLastError());
        MEL_CUDA_OK(cudaMemcpyAsync(h->h_red, h->d_red, 4 * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
        MEL_CUDA_OK(cudaStreamSynchronize(h->stream));
        if ((rc = check_errors(h))) return rc;
        mean_error = h->h_red[0]; max_error = h->h_red[1]; total_mass = h->h_red[2]; max_mass = h->h_red[3];
        const double error = max_error;
        bool reject = false;
        switch (h->solver) {
        case MEL_SOLVER_ADAPTIVE_EULER:
            reject = error > Target_error * Accepted_ratio;
            dt_law(h, error / Target_error, 1. / Accepted_ratio);
            break;
        case MEL_SOLVER_EULER_2:
            dt_law(h, error / Target_error, 1. / Accepted_ratio);
            break;
        case MEL_SOLVER_MASS_SCALING:
            reject = max_error > Target_error * Accepted_ratio;
            dt_law(h, max_error * Inv_Target_error, 1. / Accepted_ratio);
            break;
        case MEL_SOLVER_ADAPTIVE_MASS_SCALING:
            reject = max_mass > Accepted_ratio + 0.05;
            if (reject) dt_law(h, max_mass, 1. / Accepted_ratio);
            else {
                const double c2 = 1. / Accepted_ratio;
                h->dt = h->dt / pow(c2, h->d.sp[1]);
                if (h->dt > h->cup) h->dt = h->cup;
            }
            break;
        }
        if (reject) {
            // the correction above used the attempt's Deltat; Time stays
            if ((rc = adaptive_store(h, true))) return rc;
        } else {
            ok = true;
        }
        if (!ok && neval > 1000) break;
    }
    if (ok) {
        // Time += Deltat happened with the Deltat of the accepted attempt: recover it from the
        // snapshot of the attempt (h_red[7]) before the law changed h->dt
        h->time += h->h_red[7];
        h->pressure_state = 1;
    }
    h->solver_stats[0] = neval; h->solver_stats[1] = max_error; h->solver_stats[2] = mean_error;
    h->solver_stats[3] = total_mass; h->solver_stats[4] = max_mass;
    return MEL_OK;
}

// Update_contact_pressures on the handle's stream, if the last step's pressures are not computed yet
static void update_pressures(mel_handle* h)
{
    if (h->pressure_state != 1) return;
    cudaMemsetAsync(h->d.err + MEL_E_PRESSURE, 0, sizeof(unsigned), h->stream);
    mel_launch_contact_pressures(h->d, h->stream);
    h->launches += 3;
    h->pressure_state = 0;
}

extern "C" {

static mel_status create_impl(const mel_model_desc* desc, const mel_options* opt, const mel_contact* c0, int nc0,
                              mel_handle** out)
{
    if (!out) { mel_set_error("null output handle"); return MEL_ERR_INVALID; }
    *out = nullptr;
    mel_status rc = validate(desc);
    if (rc) return rc;
    if (opt && (opt->use_graph != 0 || opt->max_contacts != 0)) { mel_set_error("mel_options: use_graph and max_contacts are reserved and must be 0"); return MEL_ERR_INVALID; }
    if (opt && opt->precision != MEL_PREC_FP64 && opt->precision != MEL_PREC_MIXED) { mel_set_error("mel_options: unknown precision %d", opt->precision); return MEL_ERR_INVALID; }
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) { mel_set_error("no CUDA device"); return MEL_ERR_NO_DEVICE; }
    mel_handle* h = new mel_handle();
    h->device = opt ? opt->device : 0;
    if (cudaSetDevice(h->device) != cudaSuccess) { mel_set_error("cudaSetDevice(%d) failed", h->device); delete h; return MEL_ERR_NO_DEVICE; }
    if (cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) != cudaSuccess) { mel_set_error("stream"); delete h; return MEL_ERR_CUDA; }
    rc = build(h, desc, opt);
    h->t_bc = desc->time;                  // set-up's Update_bc(Time) (Code/main.cpp:104-127)
    if (!rc) rc = upload_state(h, desc->node_state, h->rg_file.data());
    if (!rc && nc0 > 0) rc = mel_set_contacts(h, c0, nc0);   // contacts of the DYNAMIC file (Code/IO.h:2236-2302)
    if (!rc) rc = setup(h);
    if (rc) { mel_destroy(h); return rc; }
    *out = h;
    return MEL_OK;
}

mel_status mel_create(const mel_model_desc* desc, const mel_options* opt, mel_handle** out)
{
    return create_impl(desc, opt, nullptr, 0, out);
}

mel_status mel_create_from_files(const char* dir, int restart_index, const mel_options* opt, mel_handle** out)
{
    mel_host_model hm;
    mel_status rc = mel_load_files(dir, restart_index, &hm);
    if (rc) return rc;
    return create_impl(&hm.desc, opt, hm.contacts.data(), (int)hm.contacts.size(), out);
}

/* the model read from the files, for callers that drive their own copy (returns a heap object) */
mel_status mel_load_desc(const char* dir, int restart_index, mel_model_desc** desc_out, void** owner)
{
    if (!desc_out || !owner) return MEL_ERR_INVALID;
    mel_host_model* hm = new mel_host_model();
    mel_status rc = mel_load_files(dir, restart_index, hm);
    if (rc) { delete hm; return rc; }
    *desc_out = &hm->desc;
    *owner = hm;
    return MEL_OK;
}

mel_status mel_create_loaded(const void* owner, const mel_options* opt, mel_handle** out)
{
    if (!owner || !out) { mel_set_error("invalid arguments"); return MEL_ERR_INVALID; }
    const mel_host_model* hm = static_cast<const mel_host_model*>(owner);
    return create_impl(&hm->desc, opt, hm->contacts.data(), (int)hm->contacts.size(), out);
}

mel_status mel_load_run_control(const void* owner, mel_run_control* out)
{
    if (!owner || !out) { mel_set_error("invalid arguments"); return MEL_ERR_INVALID; }
    const mel_host_model* hm = static_cast<const mel_host_model*>(owner);
    if (hm->monitored.size() > MEL_MON_MAX) {
        mel_set_error("%zu monitored entries, at most %d are supported", hm->monitored.size(), MEL_MON_MAX);
        return MEL_ERR_UNSUPPORTED;
    }
    memset(out, 0, sizeof *out);
    snprintf(out->simulation_name, sizeof out->simulation_name, "%s", hm->name.c_str());
    out->save_period = hm->save_period; out->print_period = hm->print_period;
    out->next_save = hm->next_save; out->next_print = hm->next_print;
    out->number_save = hm->number_save; out->number_iteration = hm->number_iteration; out->number_print = hm->number_print;
    out->n_monitored = (int)hm->monitored.size();
    for (size_t i = 0; i < hm->monitored.size(); i++)
        for (size_t k = 0; k < hm->monitored[i].size() && k < MEL_MON_NF; k++)
            out->monitored[MEL_MON_NF * i + k] = hm->monitored[i][k];
    for (int k = 0; k < MEL_NFLAGS; k++) out->flags[k] = hm->desc.flags[k];
    return MEL_OK;
}

mel_status mel_free_desc(void* owner)
{
    delete static_cast<mel_host_model*>(owner);
    return MEL_OK;
}

mel_status mel_destroy(mel_handle* h)
{
    if (!h) return MEL_OK;
    cudaSetDevice(h->device);
    if (h->batch) mel_batch_retire(h->batch, h);
    if (h->stream) cudaStreamSynchronize(h->stream);
    for (void* p : h->allocs) cudaFree(p);
    mel_prox_state& P = h->P;
    for (void* p : { (void*)P.nbr, (void*)P.task, (void*)P.inc_task, (void*)P.slot_cnt, (void*)P.slot_off, (void*)P.tmap, (void*)P.nzoff, (void*)P.nzlist, (void*)P.inc_rng,
                     (void*)P.scan_ws,
                     (void*)P.tns, (void*)P.tslot, (void*)P.tkey,
                     (void*)P.e_list, (void*)P.cont_alt, (void*)P.cont_w, (void*)P.cont_rt, (void*)h->d.cont })
        if (p) cudaFree(p);
    mel_prox_stage_free(P.stage);
    if (h->ck.side) { cudaStreamSynchronize(h->ck.side); cudaStreamDestroy(h->ck.side); }
    if (h->ck.packed) cudaEventDestroy(h->ck.packed);
    if (h->ck.landed) cudaEventDestroy(h->ck.landed);
    if (h->ck.d_stage) cudaFree(h->ck.d_stage);
    if (h->d_state) cudaFree(h->d_state);
    for (void* p : h->store_bufs) cudaFree(p);
    if (h->h_red) cudaFreeHost(h->h_red);
    for (void* p : { (void*)h->mon_ops, (void*)h->mon_part, (void*)h->mon_rows }) if (p) cudaFree(p);
    if (h->ck.h_stage) cudaFreeHost(h->ck.h_stage);
    for (auto e : h->ev_pool) cudaEventDestroy(e);
    if (h->ev_start) { cudaEventDestroy(h->ev_start); cudaEventDestroy(h->ev_end); }
    if (h->stream) cudaStreamDestroy(h->stream);
    delete h;
    return MEL_OK;
}

mel_status mel_step(mel_handle* h, mel_step_io* io)
{
    if (!h || !io || io->nsteps < 0) { mel_set_error("invalid arguments"); return MEL_ERR_INVALID; }
    if (h->batch) { mel_set_error("the handle is a member of a batch: step it with mel_batch_step"); return MEL_ERR_INVALID; }
    cudaSetDevice(h->device);
    h->t_contact = h->t_body = h->t_prox = h->t_total = 0.;
    h->launches = 0;
    int nprox = 0;
    // timing events: three per step, two per proximity update (at most one per step)
    size_t need = h->timing ? (size_t)5 * io->nsteps : 0;
    while (h->ev_pool.size() < need) { cudaEvent_t e; cudaEventCreate(&e); h->ev_pool.push_back(e); }
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> pev;
    if (!h->ev_start) { cudaEventCreate(&h->ev_start); cudaEventCreate(&h->ev_end); }
    cudaEventRecord(h->ev_start, h->stream);
    size_t nev = 0;
    std::vector<cudaEvent_t> ev;
    auto mark = [&]() { if (!h->timing) return; cudaEvent_t e = h->ev_pool[nev++]; cudaEventRecord(e, h->stream); ev.push_back(e); };
    std::vector<int> kinds;
    const bool adaptive = h->solver != MEL_SOLVER_EULER;
    if (h->mon_on && h->mon_count + io->nsteps > h->mon_cap) {
        mel_set_error("monitoring rows: %d recorded and %d more steps exceed the buffer of %d rows; drain them with "
                      "mel_monitor_rows first", h->mon_count, io->nsteps, h->mon_cap);
        return MEL_ERR_INVALID;
    }
    for (int s = 0; s < io->nsteps; s++) {
        if (adaptive) {
            // Solver_step (Code/Solver.h:98-486, dispatched at Code/main.cpp:156-167)
            mel_status rc = adaptive_step(h);
            if (rc) return rc;
        } else {
            mark();
            mel_launch_contact(h->d, 1.0, h->stream);
            mark(); kinds.push_back(0);
            if (h->d.fdamp) { mel_launch_damping(h->d, h->stream); h->launches++; }
            if (h->d.falid) { mel_launch_alid(h->d, h->parity, 0., 0, h->stream); h->launches++; }
            mel_launch_body(h->d, h->parity, h->nblocks_body, h->body_smem, h->stream, h->nwide);
            if (h->nwide && h->nblocks_body) h->launches++;
            mark(); kinds.push_back(1);
            {
                cudaError_t le = cudaGetLastError();
                if (le != cudaSuccess) { mel_set_cuda_error(le, "step kernel launch", __FILE__, __LINE__); return MEL_ERR_CUDA; }
            }
            h->launches += 2;
            h->parity ^= 1;
            h->time += h->dt;                       // Code/Solver.h:86
            h->pressure_state = 1;                  // Update_contact_pressures ends the step (Code/Solver.h:87)
        }
        h->iteration++;                             // Number_iteration (Code/main.cpp:143)
        if (h->mon_on) {                            // Monitoring (Code/main.cpp:173-177)
            mel_mon_head hd;
            hd.iteration = (double)h->iteration; hd.time = h->time; hd.dt = h->dt;
            hd.neval = h->solver_stats[0]; hd.max_error = h->solver_stats[1]; hd.mean_error = h->solver_stats[2];
            mel_launch_monitor(h->d, h->mon_ops, h->mon_nops, h->mon_energy, h->mon_bound, h->mon_part,
                               h->mon_rows + (size_t)h->mon_count * h->mon_stride, hd, h->stream);
            cudaError_t le = cudaGetLastError();
            if (le != cudaSuccess) { mel_set_cuda_error(le, "monitoring launch", __FILE__, __LINE__); return MEL_ERR_CUDA; }
            h->mon_count++;
            h->launches += 2;
        }
        if (io->run_proximity && h->time > h->next_cup - 1.e-6 * h->dt) {   // Code/main.cpp:191-196
            h->next_cup = h->next_cup + h->cup;
            update_pressures(h);                // from the list the step ended with
            cudaEvent_t p0 = nullptr, p1 = nullptr;
            if (h->timing) { p0 = h->ev_pool[nev++]; p1 = h->ev_pool[nev++]; pev.push_back({ p0, p1 }); }
            mel_status rc = proximity(h, p0, p1);
            if (rc) return rc;
            nprox++;
            if (h->n_deact) {                   // Update_status (Code/main.cpp:195)
                mel_launch_status(h->d, h->d_deact, h->n_deact, h->stream);
                h->launches++;
            }
        }
    }
    if (adaptive) {
        // the device clock of the Euler launches follows the host's (Time, Deltat)
        double t2[2] = { h->time, h->time };
        MEL_CUDA_OK(cudaMemcpyAsync(h->d.time2, t2, sizeof t2, cudaMemcpyHostToDevice, h->stream));
        MEL_CUDA_OK(cudaMemcpyAsync(h->d.dt, &h->dt, sizeof(double), cudaMemcpyHostToDevice, h->stream));
    }
    cudaEventRecord(h->ev_end, h->stream);
    cudaError_t e = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess) { mel_set_cuda_error(e, "mel_step", __FILE__, __LINE__); return MEL_ERR_CUDA; }
    {
        float tot = 0.f;
        cudaEventElapsedTime(&tot, h->ev_start, h->ev_end);
        h->t_total = tot;
    }
    if (h->timing) {
        for (size_t k = 0; k + 2 < ev.size(); k += 3) {
            float a = 0.f, b = 0.f;
            cudaEventElapsedTime(&a, ev[k], ev[k + 1]);
            cudaEventElapsedTime(&b, ev[k + 1], ev[k + 2]);
            h->t_contact += a; h->t_body += b;
        }
        for (auto& pe : pev) {
            float ms = 0.f;
            cudaEventElapsedTime(&ms, pe.first, pe.second);
            h->t_prox += ms;
        }
    }
    mel_status rc = check_errors(h);
    if (rc) return rc;
    io->time = h->time; io->dt = h->dt; io->next_contact_update = h->next_cup;
    io->n_contacts = h->d.ncont; io->n_proximity = nprox;
    return MEL_OK;
}

mel_status mel_update_proximity(mel_handle* h)
{
    if (!h) return MEL_ERR_INVALID;
    cudaSetDevice(h->device);
    mel_status rc = proximity(h);
    if (rc) return rc;
    if (cudaStreamSynchronize(h->stream) != cudaSuccess) { mel_set_cuda_error(cudaGetLastError(), "proximity", __FILE__, __LINE__); return MEL_ERR_CUDA; }
    return check_errors(h);
}

mel_status mel_set_contacts(mel_handle* h, const mel_contact* c, int n)
{
    if (!h || n < 0 || (n > 0 && !c)) { mel_set_error("invalid arguments"); return MEL_ERR_INVALID; }
    cudaSetDevice(h->device);
    const std::vector<int>& bb = h->H.b_bd0;
    const std::vector<int>& be = h->H.bd_e0;
    for (int i = 0; i < n; i++) {
        const mel_contact& k = c[i];
        if (k.bodyS < 0 || k.bodyS >= h->nb || k.bodyM < 0 || k.bodyM >= h->nb) { mel_set_error("contact %d: body out of range", i); return MEL_ERR_INVALID; }
        if (i > 0 && k.bodyS < c[i - 1].bodyS) { mel_set_error("contact list must be ordered by slave body"); return MEL_ERR_INVALID; }
        int nbS = bb[k.bodyS + 1] - bb[k.bodyS], nbM = bb[k.bodyM + 1] - bb[k.bodyM];
        if (k.borderS < 0 || k.borderS >= nbS || k.borderM < 0 || k.borderM >= nbM) { mel_set_error("contact %d: border out of range", i); return MEL_ERR_INVALID; }
        int gS = bb[k.bodyS] + k.borderS, gM = bb[k.bodyM] + k.borderM;
        if (k.border_nodeS < 0 || k.border_nodeS >= be[gS + 1] - be[gS]) { mel_set_error("contact %d: border node out of range", i); return MEL_ERR_INVALID; }
        if (k.segmentM < 0 || k.segmentM > be[gM + 1] - be[gM] - 2) { mel_set_error("contact %d: segment out of range", i); return MEL_ERR_INVALID; }
        int nnS = h->b_node0[k.bodyS + 1] - h->b_node0[k.bodyS];
        if (k.nodeS < 0 || k.nodeS >= nnS) { mel_set_error("contact %d: slave node out of range", i); return MEL_ERR_INVALID; }
    }
    size_t need = sizeof(mel_contact) * (size_t)(n + 1);
    if (need > h->P.cont_bytes) {
        cudaFree(h->d.cont);
        if (cudaMalloc(&h->d.cont, need) != cudaSuccess) return MEL_ERR_OOM;
        h->P.cont_bytes = need;
    }
    if (sizeof(double) * (size_t)(n + 1) > h->P.cont_w_bytes) {
        cudaFree(h->P.cont_w);
        if (cudaMalloc(&h->P.cont_w, sizeof(double) * (n + 1)) != cudaSuccess) return MEL_ERR_OOM;
        h->P.cont_w_bytes = sizeof(double) * (n + 1);
    }
    h->d.cont_w = h->P.cont_w;
    cudaMemset(h->P.cont_w, 0, sizeof(double) * (n + 1));
    if (6 * sizeof(double) * (size_t)(n + 1) > h->P.cont_rt_bytes) {
        cudaFree(h->P.cont_rt);
        if (cudaMalloc(&h->P.cont_rt, 6 * sizeof(double) * (n + 1)) != cudaSuccess) return MEL_ERR_OOM;
        h->P.cont_rt_bytes = 6 * sizeof(double) * (n + 1);
    }
    h->d.cont_rt = h->P.cont_rt;
    if (n) MEL_CUDA_OK(cudaMemcpy(h->d.cont, c, sizeof(mel_contact) * n, cudaMemcpyHostToDevice));
    h->d.ncont = n;
    int rc = mel_index_external(h->d, h->P, c, n, h->stream);
    if (rc) return (mel_status)rc;
    return check_errors(h);
}

// node state in the 12-doubles-per-node layout of mel_model_desc::node_state
static __global__ void state_pack_kernel(const double2* u, const double2* v, const double2* a, const double2* up,
                                         const double2* vp, const double2* ap, int nn, double* out)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nn) return;
    const double2 w[6] = { u[i], v[i], a[i], up[i], vp[i], ap[i] };
    double* o = out + 12 * (size_t)i;
#pragma unroll
    for (int k = 0; k < 6; k++) { o[2 * k] = w[k].x; o[2 * k + 1] = w[k].y; }
}

// The inverse, with the positions that follow from it: deformable nodes x = X0 + u
// (Code/Node.h:233-237); rigid nodes take position and velocity from their body's state
// (Code/Body.h:2284-2300), as upload_state computes them on the host.
static __global__ void state_unpack_kernel(mel_dev d, const double* st)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= d.nn) return;
    int lo = 0, hi = d.nb;                    // body of node i: largest b with b_node0[b] <= i
    while (hi - lo > 1) { const int mid = (lo + hi) >> 1; if (d.b_node0[mid] <= i) lo = mid; else hi = mid; }
    const double* s = st + 12 * (size_t)i;
    const double2 u = make_double2(s[0], s[1]);
    double2 v = make_double2(s[2], s[3]);
    d.u[i] = u; d.a[i] = make_double2(s[4], s[5]);
    d.up[i] = make_double2(s[6], s[7]); d.vp[i] = make_double2(s[8], s[9]); d.ap[i] = make_double2(s[10], s[11]);
    const double2 X = d.X0[i];
    double2 x = make_double2(X.x + u.x, X.y + u.y);
    if (d.b_type[lo] == MEL_BODY_RIGID) {
        double* r = d.rg + MEL_RIGID_NF * lo;
        const double xc = r[MEL_RG_X0] + r[MEL_RG_XD], yc = r[MEL_RG_Y0] + r[MEL_RG_YD];
        const double dr = r[MEL_RG_RD] - r[MEL_RG_R0];
        const double dx = X.x - r[MEL_RG_X0], dy = X.y - r[MEL_RG_Y0];
        x.x = xc + dx * mel_cos(dr) - dy * mel_sin(dr);
        x.y = yc + dx * mel_sin(dr) + dy * mel_cos(dr);
        const double ddx = x.x - xc, ddy = x.y - yc;
        v = make_double2(-ddy * r[MEL_RG_RV] + r[MEL_RG_XV], ddx * r[MEL_RG_RV] + r[MEL_RG_YV]);
        if (i == d.b_node0[lo]) { r[MEL_RG_XC] = xc; r[MEL_RG_YC] = yc; r[MEL_RG_RC] = r[MEL_RG_R0] + r[MEL_RG_RD]; }
    }
    d.v[i] = v;
    d.x[i] = x;
}

static mel_status state_stage(mel_handle* h)
{
    if (h->d_state) return MEL_OK;
    if (cudaMalloc(&h->d_state, sizeof(double) * 12 * (size_t)(h->nn > 0 ? h->nn : 1)) != cudaSuccess) {
        h->d_state = nullptr;
        mel_set_error("node-state staging allocation failed");
        return MEL_ERR_OOM;
    }
    return MEL_OK;
}

// Both directions go through one device staging array in the caller's layout: one copy of
// 96 bytes per node each way (at full link speed when the caller's buffer is pinned), packed and
// unpacked by a kernel.
mel_status mel_get_node_state(mel_handle* h, double* st)
{
    if (!h || !st) return MEL_ERR_INVALID;
    cudaSetDevice(h->device);
    mel_status rc = state_stage(h);
    if (rc) return rc;
    const int nn = h->nn;
    if (nn > 0) {
        state_pack_kernel<<<(nn + 255) / 256, 256, 0, h->stream>>>(h->d.u, h->d.v, h->d.a, h->d.up, h->d.vp, h->d.ap, nn, h->d_state);
        MEL_CUDA_OK(cudaGetLastError());
        MEL_CUDA_OK(cudaMemcpyAsync(st, h->d_state, sizeof(double) * 12 * (size_t)nn, cudaMemcpyDeviceToHost, h->stream));
    }
    MEL_CUDA_OK(cudaStreamSynchronize(h->stream));
    return MEL_OK;
}

mel_status mel_set_node_state(mel_handle* h, const double* st)
{
    if (!h || !st) return MEL_ERR_INVALID;
    cudaSetDevice(h->device);
    mel_status rc = state_stage(h);
    if (rc) return rc;
    const int nn = h->nn;
    if (nn > 0) {
        MEL_CUDA_OK(cudaMemcpyAsync(h->d_state, st, sizeof(double) * 12 * (size_t)nn, cudaMemcpyHostToDevice, h->stream));
        state_unpack_kernel<<<(nn + 255) / 256, 256, 0, h->stream>>>(h->d, h->d_state);
        MEL_CUDA_OK(cudaGetLastError());
    }
    MEL_CUDA_OK(cudaStreamSynchronize(h->stream));
    return MEL_OK;
}

mel_status mel_pin_host(void* ptr, size_t bytes)
{
    if (!ptr || bytes == 0) { mel_set_error("mel_pin_host: null pointer or zero size"); return MEL_ERR_INVALID; }
    MEL_CUDA_OK(cudaHostRegister(ptr, bytes, cudaHostRegisterDefault));
    return MEL_OK;
}

mel_status mel_unpin_host(void* ptr)
{
    if (!ptr) { mel_set_error("mel_unpin_host: null pointer"); return MEL_ERR_INVALID; }
    MEL_CUDA_OK(cudaHostUnregister(ptr));
    return MEL_OK;
}

mel_status mel_set_rigid(mel_handle* h, const double* rigid)
{
    if (!h || !rigid) return MEL_ERR_INVALID;
    cudaSetDevice(h->device);
    cudaStreamSynchronize(h->stream);
    return upload_state(h, nullptr, rigid);
}

mel_status mel_set_time(mel_handle* h, double time, double dt, double next_contact_update)
{
    if (!h || !(dt > 0.)) return MEL_ERR_INVALID;
    cudaSetDevice(h->device);
    cudaStreamSynchronize(h->stream);
    h->time = time; h->dt = dt; h->next_cup = next_contact_update;
    h->t_bc = time;
    mel_launch_drivendof(h->d, time, h->stream);
    MEL_CUDA_OK(cudaGetLastError());
    MEL_CUDA_OK(cudaStreamSynchronize(h->stream));
    double t2[2] = { time, time };
    MEL_CUDA_OK(cudaMemcpy(h->d.time2, t2, sizeof t2, cudaMemcpyHostToDevice));
    MEL_CUDA_OK(cudaMemcpy(h->d.dt, &dt, sizeof dt, cudaMemcpyHostToDevice));
    h->parity = 0;
    return MEL_OK;
}

mel_status mel_get_positions(mel_handle* h, double* xy)
{
    if (!h || !xy) return MEL_ERR_INVALID;
    cudaSetDevice(h->device);
    cudaStreamSynchronize(h->stream);
    MEL_CUDA_OK(cudaMemcpy(xy, h->d.x, sizeof(double) * 2 * (size_t)h->nn, cudaMemcpyDeviceToHost));
    return MEL_OK;
}

mel_status mel_get_forces(mel_handle* h, double* internal, double* contact, double* neumann, double* dirichlet, double* total)
{
    if (!h) return MEL_ERR_INVALID;
    cudaSetDevice(h->device);
    cudaStreamSynchronize(h->stream);
    if (!h->d.record_forces) { mel_set_error("force recording is off: call mel_record_forces(h, 1) before stepping"); return MEL_ERR_INVALID; }
    size_t b = sizeof(double) * 2 * (size_t)h->nn;
    if (internal) MEL_CUDA_OK(cudaMemcpy(internal, h->d.o_fint, b, cudaMemcpyDeviceToHost));
    if (contact) MEL_CUDA_OK(cudaMemcpy(contact, h->d.o_fcon, b, cudaMemcpyDeviceToHost));
    if (neumann) MEL_CUDA_OK(cudaMemcpy(neumann, h->d.o_fneu, b, cudaMemcpyDeviceToHost));
    if (dirichlet) MEL_CUDA_OK(cudaMemcpy(dirichlet, h->d.o_fdir, b, cudaMemcpyDeviceToHost));
    if (total) MEL_CUDA_OK(cudaMemcpy(total, h->d.o_ftot, b, cudaMemcpyDeviceToHost));
    return MEL_OK;
}

mel_status mel_record_forces(mel_handle* h, int on)
{
    if (!h) return MEL_ERR_INVALID;
    h->d.record_forces = (on || h->mon_forces || h->deact_forces) ? 1 : 0;   // force entries keep it on
    return MEL_OK;
}

mel_status mel_set_timing(mel_handle* h, int on)
{
    if (!h) return MEL_ERR_INVALID;
    h->timing = on ? 1 : 0;
    return MEL_OK;
}

mel_status mel_get_rigid(mel_handle* h, double* rigid, double* rigid_forces)
{
    if (!h) return MEL_ERR_INVALID;
    cudaSetDevice(h->device);
    cudaStreamSynchronize(h->stream);
    if (rigid) MEL_CUDA_OK(cudaMemcpy(rigid, h->d.rg, sizeof(double) * MEL_RIGID_NF * (size_t)h->nb, cudaMemcpyDeviceToHost));
    if (rigid_forces) {
        std::vector<double> rf(15 * (size_t)h->nb);
        MEL_CUDA_OK(cudaMemcpy(rf.data(), h->d.rf, sizeof(double) * rf.size(), cudaMemcpyDeviceToHost));
        for (int b = 0; b < h->nb; b++) memcpy(rigid_forces + 12 * (size_t)b, &rf[15 * (size_t)b], 12 * sizeof(double));
    }
    return MEL_OK;
}

mel_status mel_get_works(mel_handle* h, double* works)
{
    if (!h || !works) return MEL_ERR_INVALID;
    cudaSetDevice(h->device);
    cudaStreamSynchronize(h->stream);
    MEL_CUDA_OK(cudaMemcpy(works, h->d.works, sizeof(double) * 7 * (size_t)h->nb, cudaMemcpyDeviceToHost));
    return MEL_OK;
}

mel_status mel_get_contact_pressures(mel_handle* h, double* px, double* py)
{
    if (!h || (!px && !py)) { mel_set_error("invalid arguments"); return MEL_ERR_INVALID; }
    cudaSetDevice(h->device);
    if (h->pressure_state == 2) {
        mel_set_error("the contact list changed since the last step: a batch member keeps its contact pressures only "
                      "with mel_record_forces on");
        return MEL_ERR_INVALID;
    }
    update_pressures(h);
    MEL_CUDA_OK(cudaStreamSynchronize(h->stream));
    if (h->ne > 0) {
        if (px) MEL_CUDA_OK(cudaMemcpy(px, h->d.cpx, sizeof(double) * (size_t)h->ne, cudaMemcpyDeviceToHost));
        if (py) MEL_CUDA_OK(cudaMemcpy(py, h->d.cpy, sizeof(double) * (size_t)h->ne, cudaMemcpyDeviceToHost));
    }
    // an output-only quantity: an entry with more contributions than the gather holds fails this
    // call (its pressure would be incomplete), never a step
    unsigned w[MEL_E_NWORDS];
    MEL_CUDA_OK(cudaMemcpy(w, h->d.err, sizeof w, cudaMemcpyDeviceToHost));
    if (w[MEL_E_PRESSURE]) {
        mel_set_error("a border entry gathers more than %d contact contributions to its pressure", MEL_PRESSURE_CAP);
        return MEL_ERR_BOUNDS;
    }
    return check_errors(h);
}

mel_status mel_get_solver_stats(mel_handle* h, double* out5)
{
    if (!h || !out5) { mel_set_error("invalid arguments"); return MEL_ERR_INVALID; }
    for (int k = 0; k < 5; k++) out5[k] = h->solver_stats[k];
    return MEL_OK;
}

mel_status mel_get_contact_count(mel_handle* h, int* n)
{
    if (!h || !n) return MEL_ERR_INVALID;
    *n = h->d.ncont;
    return MEL_OK;
}

mel_status mel_get_contacts(mel_handle* h, mel_contact* out, int capacity, int* n)
{
    if (!h) return MEL_ERR_INVALID;
    cudaSetDevice(h->device);
    cudaStreamSynchronize(h->stream);
    if (n) *n = h->d.ncont;
    int m = std::min(capacity, h->d.ncont);
    if (out && m > 0) MEL_CUDA_OK(cudaMemcpy(out, h->d.cont, sizeof(mel_contact) * m, cudaMemcpyDeviceToHost));
    return MEL_OK;
}

mel_status mel_get_body_status(mel_handle* h, int* status)
{
    if (!h || !status) { mel_set_error("invalid arguments"); return MEL_ERR_INVALID; }
    cudaSetDevice(h->device);
    MEL_CUDA_OK(cudaStreamSynchronize(h->stream));
    MEL_CUDA_OK(cudaMemcpy(status, h->d.b_status, sizeof(int) * (size_t)h->nb, cudaMemcpyDeviceToHost));
    return MEL_OK;
}

mel_status mel_get_bc_pressures(mel_handle* h, double* px, double* py)
{
    if (!h || (!px && !py)) { mel_set_error("invalid arguments"); return MEL_ERR_INVALID; }
    cudaSetDevice(h->device);
    MEL_CUDA_OK(cudaStreamSynchronize(h->stream));
    if (h->ne > 0) {
        std::vector<double2> p(h->ne);
        MEL_CUDA_OK(cudaMemcpy(p.data(), h->d.e_bcp, sizeof(double2) * (size_t)h->ne, cudaMemcpyDeviceToHost));
        for (int e = 0; e < h->ne; e++) { if (px) px[e] = p[e].x; if (py) py[e] = p[e].y; }
    }
    return MEL_OK;
}

// ---------------------------------------------------------------------------------------------
// Monitoring on the device (Code/Monitoring.h:8-559, rows drained as Write_monitoring flushes them)
// ---------------------------------------------------------------------------------------------
mel_status mel_monitor_setup(mel_handle* h, const double* monitored, int n_monitored, int monitor_energy,
                             int monitor_boundaries, int ring_rows, int first_iteration, int* max_row_length)
{
    if (!h || n_monitored < 0 || ring_rows < 0 || (n_monitored > 0 && !monitored)) { mel_set_error("invalid arguments"); return MEL_ERR_INVALID; }
    if (h->batch) { mel_set_error("monitoring runs on handles stepped with mel_step, not on batch members"); return MEL_ERR_INVALID; }
    cudaSetDevice(h->device);
    MEL_CUDA_OK(cudaStreamSynchronize(h->stream));
    const bool on = n_monitored > 0 || monitor_energy || monitor_boundaries;
    if (on && ring_rows == 0) { mel_set_error("monitoring needs a row buffer (ring_rows > 0)"); return MEL_ERR_INVALID; }
    // the entries as the kernel reads them, checked against the model (the reference indexes its
    // arrays with them unchecked)
    std::vector<int> nodes_of(h->nb);
    for (int b = 0; b < h->nb; b++) nodes_of[b] = h->b_node0[b + 1] - h->b_node0[b];
    std::vector<int> bd0(h->nb + 1);
    MEL_CUDA_OK(cudaMemcpy(bd0.data(), h->d.b_bd0, sizeof(int) * (h->nb + 1), cudaMemcpyDeviceToHost));
    std::vector<mel_mon_op> ops;
    int row = 6;
    bool forces = false;
    for (int i = 0; i < n_monitored; i++) {
        const double* e = monitored + (size_t)MEL_MON_NF * i;
        mel_mon_op o;
        memset(&o, 0, sizeof o);
        o.type = (int)e[0];
        o.node = -1;
        auto body_ok = [&](int b) { return b >= 0 && b < h->nb; };
        auto bad = [&](const char* what) {
            mel_set_error("monitored entry %d (type %d): %s", i, o.type, what);
            return MEL_ERR_INVALID;
        };
        if (o.type >= 0 && o.type <= 3) {
            o.kind = (int)e[1]; o.body = (int)e[2]; o.node = (int)e[3];
            if (o.type == 0 && o.kind >= 3) continue;    // Length / Area / AllX / AllY: spies only
            if (!body_ok(o.body) || o.node >= nodes_of[o.body]) return bad("body or node out of range");
            if (o.kind >= 0 && o.kind <= (o.type == 0 ? 2 : 3)) row++;
        } else if (o.type == 4) {
            o.kind = (int)e[1]; o.sub = (int)e[2]; o.body = (int)e[3]; o.node = (int)e[4];
            if (!body_ok(o.body) || o.node >= nodes_of[o.body] || o.sub < 0 || o.sub > 7) return bad("body, node or force kind out of range");
            if (o.node < 0 && h->b_type[o.body] == MEL_BODY_DEFORMABLE) {
                // Code/Monitoring.h:232 walks as many nodes as body number `sub` has
                if (o.sub >= h->nb || nodes_of[o.sub] > nodes_of[o.body])
                    return bad("the reference sums over as many nodes as body number <force kind> has, more than the body holds");
            }
            if (o.node >= 0 || h->b_type[o.body] == MEL_BODY_DEFORMABLE) forces = true;
            if (o.kind >= 0 && o.kind <= 3) row++;
        } else if (o.type == 5 || o.type == 6) {
            mel_set_error("monitored entry %d: type %d (%s) needs the nodal stress post-processing (Code/Body.h:2310-2519), "
                          "which this library does not run", i, o.type, o.type == 5 ? "Jacobian" : "Stress");
            return MEL_ERR_UNSUPPORTED;
        } else if (o.type == 8) {
            o.body = (int)e[1];                          // Damage: Update_damage of the body
            if (!body_ok(o.body)) return bad("body out of range");
            row++;
        } else if (o.type == 7) {
            o.kind = (int)e[1]; o.body = (int)e[2]; o.border = (int)e[3]; o.bnode = (int)e[4];
            if (!body_ok(o.body)) return bad("body out of range");
            // a value only while that slave node has a contact element: rows vary in length
            if (o.kind >= 0 && o.kind <= 5) row++;
        } else if (o.type == 9) {
            o.kind = (int)e[1]; o.body = (int)e[2];
            if (o.body >= h->nb || o.body < -1) return bad("body out of range");
            row++;
        } else if (o.type == 10) {
            o.kind = (int)e[1]; o.body = (int)e[2];
            if (o.body >= h->nb || o.body < -1) return bad("body out of range");
            if (o.body == -1 || (o.kind >= 0 && o.kind < 7)) row++;
        } else {
            continue;                                    // types Monitoring ignores add no column
        }
        ops.push_back(o);
    }
    if (monitor_energy) row += 3;
    if (monitor_boundaries) {
        if (h->nb < 2 || bd0[1] - bd0[0] < 1 || bd0[2] - bd0[1] < 2) {
            mel_set_error("MONITOR_BOUNDARIES reads border 0 of body 0 and border 1 of body 1, which this model lacks");
            return MEL_ERR_INVALID;
        }
        row += 4;
    }
    for (void* p : { (void*)h->mon_ops, (void*)h->mon_part, (void*)h->mon_rows }) if (p) cudaFree(p);
    h->mon_ops = nullptr; h->mon_part = nullptr; h->mon_rows = nullptr;
    h->mon_on = false; h->mon_forces = false; h->mon_count = 0; h->mon_cap = 0; h->mon_nops = 0;
    if (max_row_length) *max_row_length = on ? row : 0;
    h->iteration = first_iteration;
    if (!on) return MEL_OK;
    const size_t stride = (size_t)row + 1;
    if (cudaMalloc(&h->mon_ops, sizeof(mel_mon_op) * (ops.size() + 1)) != cudaSuccess ||
        cudaMalloc(&h->mon_part, sizeof(double) * 3 * ((size_t)h->nb + 1)) != cudaSuccess ||
        cudaMalloc(&h->mon_rows, sizeof(double) * stride * (size_t)ring_rows) != cudaSuccess) {
        for (void* p : { (void*)h->mon_ops, (void*)h->mon_part, (void*)h->mon_rows }) if (p) cudaFree(p);
        h->mon_ops = nullptr; h->mon_part = nullptr; h->mon_rows = nullptr;
        mel_set_error("monitoring buffers (%d rows of %d values) could not be allocated", ring_rows, row);
        return MEL_ERR_OOM;
    }
    if (!ops.empty()) MEL_CUDA_OK(cudaMemcpy(h->mon_ops, ops.data(), sizeof(mel_mon_op) * ops.size(), cudaMemcpyHostToDevice));
    h->mon_nops = (int)ops.size();
    h->mon_energy = monitor_energy ? 1 : 0;
    h->mon_bound = monitor_boundaries ? 1 : 0;
    h->mon_stride = (int)stride;
    h->mon_cap = ring_rows;
    h->mon_on = true;
    h->mon_forces = forces;
    if (forces) h->d.record_forces = 1;
    return MEL_OK;
}

mel_status mel_monitor_rows(mel_handle* h, double* rows, int max_rows, int* n_rows)
{
    if (!h || !n_rows || max_rows < 0) { mel_set_error("invalid arguments"); return MEL_ERR_INVALID; }
    cudaSetDevice(h->device);
    MEL_CUDA_OK(cudaStreamSynchronize(h->stream));
    *n_rows = h->mon_count;
    if (h->mon_count == 0 || (!rows && max_rows == 0)) return MEL_OK;    // nothing held, or a count query
    if (!rows || max_rows < h->mon_count) {
        mel_set_error("%d monitoring rows are recorded, the buffer holds %d", h->mon_count, max_rows);
        return MEL_ERR_INVALID;
    }
    MEL_CUDA_OK(cudaMemcpy(rows, h->mon_rows, sizeof(double) * (size_t)h->mon_stride * h->mon_count, cudaMemcpyDeviceToHost));
    h->mon_count = 0;
    return MEL_OK;
}

// ---------------------------------------------------------------------------------------------
// Write_dynamic (Code/IO.h:2351-2640): the reference's restart file from the device state
// ---------------------------------------------------------------------------------------------
mel_status mel_write_dynamic(mel_handle* h, const char* dir, const mel_save_info* info)
{
    if (!h || !dir || !info) { mel_set_error("invalid arguments"); return MEL_ERR_INVALID; }
    if (info->number_save < 0 || info->number_save >= 100000) { mel_set_error("number_save %d outside 0..99999", info->number_save); return MEL_ERR_INVALID; }
    cudaSetDevice(h->device);
    if (!h->d.record_forces) {
        mel_set_error("the FORCES blocks need the nodal forces of the last step: call mel_record_forces(h, 1) before it");
        return MEL_ERR_INVALID;
    }
    if (h->pressure_state == 2) {
        mel_set_error("the contact list changed since the last step: its contact pressures are gone");
        return MEL_ERR_INVALID;
    }
    update_pressures(h);
    MEL_CUDA_OK(cudaStreamSynchronize(h->stream));
    const size_t nn = (size_t)h->nn, nb = (size_t)h->nb, ne = (size_t)h->ne, nbd = (size_t)h->nbd;
    const mel_dev& D = h->d;
    auto get = [&](auto* dst, const auto* src, size_t n) {
        return n ? cudaMemcpy(dst, src, sizeof(*dst) * n, cudaMemcpyDeviceToHost) : cudaSuccess;
    };
    std::vector<double2> x(nn), u(nn), v(nn), a(nn), up(nn), vp(nn), ap(nn), mass(nn);
    std::vector<double2> fint(nn), fcon(nn), fneu(nn), fdir(nn), ftot(nn), bcp(ne), fdmp(nn, make_double2(0., 0.));
    std::vector<double> rg(MEL_RIGID_NF * nb), rf(15 * nb), rtot(3 * nb), works(7 * nb), len(ne), cpx(ne), cpy(ne);
    std::vector<int> bd0(nb + 1), e0(nbd + 1), sn(4 * ne), ss(4 * ne), nbn(nb), cont0(nb + 1);
    std::vector<mel_contact> cont(D.ncont);
    const double2* srcs[] = { D.x, D.u, D.v, D.a, D.up, D.vp, D.ap, D.mass, D.o_fint, D.o_fcon, D.o_fneu, D.o_fdir, D.o_ftot };
    std::vector<double2>* dsts[] = { &x, &u, &v, &a, &up, &vp, &ap, &mass, &fint, &fcon, &fneu, &fdir, &ftot };
    for (int k = 0; k < 13; k++) MEL_CUDA_OK(get(dsts[k]->data(), srcs[k], nn));
    MEL_CUDA_OK(get(bcp.data(), D.e_bcp, ne));
    if (D.fdamp) MEL_CUDA_OK(get(fdmp.data(), D.fdamp, nn));
    MEL_CUDA_OK(get(rg.data(), D.rg, rg.size()));
    MEL_CUDA_OK(get(rf.data(), D.rf, rf.size()));
    MEL_CUDA_OK(get(rtot.data(), D.rtot, rtot.size()));
    MEL_CUDA_OK(get(works.data(), D.works, works.size()));
    MEL_CUDA_OK(get(len.data(), D.e_len, ne));
    MEL_CUDA_OK(get(cpx.data(), D.cpx, ne));
    MEL_CUDA_OK(get(cpy.data(), D.cpy, ne));
    MEL_CUDA_OK(get(bd0.data(), D.b_bd0, nb + 1));
    MEL_CUDA_OK(get(e0.data(), D.bd_e0, nbd + 1));
    MEL_CUDA_OK(get(sn.data(), D.e_sn, 4 * ne));
    MEL_CUDA_OK(get(ss.data(), D.e_ss, 4 * ne));
    MEL_CUDA_OK(get(cont0.data(), D.b_cont0, nb + 1));
    std::vector<int> status(nb);
    MEL_CUDA_OK(get(status.data(), (const int*)D.b_status, nb));
    MEL_CUDA_OK(get(cont.data(), D.cont, (size_t)D.ncont));
    std::vector<int> nbr;
    if (h->P.nbr && h->P.nbn) {
        MEL_CUDA_OK(get(nbn.data(), h->P.nbn, nb));
        nbr.resize((size_t)3 * h->P.nbr_cap * nb);
        MEL_CUDA_OK(get(nbr.data(), h->P.nbr, nbr.size()));
    }
    static const char* solver_names[] = { "Euler", "Adaptive_Euler", "Mass_Scaling", "Adaptive_Mass_Scaling", "Euler_2" };
    static const char* status_names[] = { "active", "inactive", "nogravity" };
    char fname[64];
    snprintf(fname, sizeof fname, "/DYNAMIC_%05d.asc", info->number_save);
    const std::string path = std::string(dir) + fname;
    std::ofstream F(path);
    if (!F) { mel_set_error("cannot write %s", path.c_str()); return MEL_ERR_IO; }
    const char* bar = "%%%%%%%%%%%%%%%%%%%%%%%%%%%%%%%%%%%%%%%%%%%%%%";
    F << std::endl << bar << std::endl << "%%%%%%%          GENERAL DATA          %%%%%%%" << std::endl << bar << std::endl << std::endl;
    F << "SIMULATION_NAME" << std::endl << (info->simulation_name ? info->simulation_name : "") << std::endl << std::endl;
    F << "SOLVER" << std::endl << solver_names[h->solver] << std::endl;
    F << std::setprecision(16) << info->number_save << ' ' << info->number_iteration << ' ' << h->time << ' ' << info->number_print << std::endl;
    F << std::setprecision(10) << h->dt << std::endl;       // this precision holds for the rest of the file
    F << info->next_save << ' ' << info->next_print << ' ' << h->next_cup << std::endl << std::endl;
    const char* flag_lines[MEL_NFLAGS] = { nullptr, "MONITOR_ENERGY", "MONITOR_BOUNDARIES", nullptr, "UPDATE_MASS_MATRIX",
                                           "UPDATE_STIFFNESS_MATRIX", "UPDATE_DAMPING_MATRIX", "NO_LOG", "NO_MONITORING",
                                           "NO_SELF_CONTACT", nullptr };
    for (int k = 0; k < MEL_NFLAGS; k++) if (flag_lines[k] && h->flags[k] == 1) F << flag_lines[k] << std::endl;
    F << std::endl;
    for (size_t i = 0; i < nb; i++) {
        const int n0 = h->b_node0[i], nbn_i = h->b_node0[i + 1] - n0;
        const bool def = h->b_type[i] == MEL_BODY_DEFORMABLE;
        const int st = status[i] >= 0 && status[i] <= 2 ? status[i] : 0;
        F << bar << std::endl << "%%%%%%%             BODY " << i << "             %%%%%%%" << std::endl << bar << std::endl << std::endl;
        F << (def ? "DEFORMABLE" : "RIGID") << std::endl << status_names[st] << std::endl << i << std::endl << std::endl;
        F << "KINEMATICS" << std::endl;
        if (def) {
            F << nbn_i << std::endl;
            for (int j = 0; j < nbn_i; j++) {
                const size_t q = (size_t)n0 + j;
                F << j << ' ' << x[q].x << ' ' << x[q].y << ' ' << u[q].x << ' ' << u[q].y << ' ' << v[q].x << ' ' << v[q].y << ' '
                  << a[q].x << ' ' << a[q].y << ' ' << up[q].x << ' ' << up[q].y << ' ' << vp[q].x << ' ' << vp[q].y << ' '
                  << ap[q].x << ' ' << ap[q].y << std::endl;
            }
            F << std::endl << "FORCES" << std::endl;
            const bool ng = h->b_status[i] == MEL_STATUS_NOGRAVITY;
            const double gx = ng ? 0. : D.gx, gy = ng ? 0. : D.gy;
            for (int j = 0; j < nbn_i; j++) {
                const size_t q = (size_t)n0 + j;
                // self-contact: zero (the reference never fills those components)
                F << j << ' ' << fint[q].x << ' ' << fint[q].y << ' ' << fcon[q].x << ' ' << fcon[q].y << ' ' << 0. << ' ' << 0. << ' '
                  << mass[q].x * gx << ' ' << mass[q].y * gy << ' ' << fdir[q].x << ' ' << fdir[q].y << ' '
                  << fneu[q].x << ' ' << fneu[q].y << ' ' << fdmp[q].x << ' ' << fdmp[q].y << ' ' << ftot[q].x << ' ' << ftot[q].y << std::endl;
            }
            F << std::endl;
        } else {
            const double* r = &rg[MEL_RIGID_NF * i];
            const double* f = &rf[15 * i];
            F << r[MEL_RG_XC] << ' ' << r[MEL_RG_YC] << ' ' << r[MEL_RG_RC] << std::endl;
            F << r[MEL_RG_XD] << ' ' << r[MEL_RG_YD] << ' ' << r[MEL_RG_RD] << std::endl;
            F << r[MEL_RG_XV] << ' ' << r[MEL_RG_YV] << ' ' << r[MEL_RG_RV] << std::endl << std::endl;
            F << "FORCES" << std::endl;
            for (int k = 0; k < 5; k++) F << f[3 * k] << ' ' << f[3 * k + 1] << ' ' << f[3 * k + 2] << std::endl;
            F << rtot[3 * i] << ' ' << rtot[3 * i + 1] << ' ' << rtot[3 * i + 2] << std::endl << std::endl;
        }
        const double* w = &works[7 * i];
        F << "WORKS" << std::endl << w[0] << ' ' << w[1] << ' ' << w[2] << ' ' << w[3] << ' ' << w[4] << ' ' << w[5] << ' ' << w[6]
          << std::endl << std::endl;
        F << "NEIGHBOURS" << std::endl;
        const int nnb = nbr.empty() ? 0 : nbn[i];
        F << nnb << std::endl;
        for (int j = 0; j < nnb; j++) {
            const int* q = &nbr[(size_t)3 * h->P.nbr_cap * i + 3 * j];
            F << q[0] << ' ' << q[1] << ' ' << q[2] << std::endl;
        }
        F << std::endl << "BORDERS" << std::endl << std::endl;
        for (int g = bd0[i]; g < bd0[i + 1]; g++) {
            F << g - bd0[i] << std::endl << e0[g + 1] - e0[g] << std::endl;
            for (int e = e0[g]; e < e0[g + 1]; e++) {
                F << len[e] << ' ';
                F << sn[4 * e] << ' ' << ss[4 * e] << ' ' << sn[4 * e + 1] << ' ' << ss[4 * e + 1] << ' ';
                F << sn[4 * e + 2] << ' ' << ss[4 * e + 2] << ' ' << sn[4 * e + 3] << ' ' << ss[4 * e + 3] << std::endl;
            }
            F << std::endl;
        }
        F << "CONTACTS" << std::endl << cont0[i + 1] - cont0[i] << std::endl;
        for (int k = cont0[i]; k < cont0[i + 1]; k++) {
            const mel_contact& c = cont[k];
            F << c.borderS << ' ' << c.border_nodeS << ' ' << c.nodeS << ' ';
            F << c.bodyM << ' ' << c.borderM << ' ' << c.shiftM << ' ' << c.segmentM << ' ';
            F << c.gapn << ' ' << c.gapt << ' ' << c.xsi << ' ';
            F << c.xnorm << ' ' << c.ynorm << ' ' << c.xtan << ' ' << c.ytan << ' ';
            F << c.length << ' ' << c.fx << ' ' << c.fy << ' ';
            for (int q = 0; q < 4; q++) F << c.nodeM[q] << ' ' << c.shapeM[q] << ' ' << c.shiftMk[q] << ' ';
            F << c.effective_mass << ' ' << c.nb_internal;
            for (int q = 0; q < c.nb_internal && q < MEL_NINTERNAL; q++) F << ' ' << c.internal[q];
            F << std::endl;
        }
        F << std::endl << "CONTACT_PRESSURES" << std::endl << std::endl;
        for (int g = bd0[i]; g < bd0[i + 1]; g++) {
            F << g - bd0[i] << std::endl << e0[g + 1] - e0[g] << std::endl;
            for (int e = e0[g]; e < e0[g + 1]; e++) F << cpx[e] << ' ' << cpy[e] << std::endl;
            F << std::endl;
        }
        F << std::endl << "BC_PRESSURES" << std::endl << std::endl;
        for (int g = bd0[i]; g < bd0[i + 1]; g++) {
            F << g - bd0[i] << std::endl << e0[g + 1] - e0[g] << std::endl;
            for (int e = e0[g]; e < e0[g + 1]; e++) F << bcp[e].x << ' ' << bcp[e].y << std::endl;
            F << std::endl;
        }
        F << std::endl;
    }
    F.close();
    if (!F) { mel_set_error("writing %s failed", path.c_str()); return MEL_ERR_IO; }
    return MEL_OK;
}

// node state in the 12-doubles-per-node layout of mel_model_desc::node_state
static __global__ void ckpt_pack_nodes(const double2* u, const double2* v, const double2* a, const double2* up,
                                       const double2* vp, const double2* ap, int nn, double* out)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nn) return;
    const double2 w[6] = { u[i], v[i], a[i], up[i], vp[i], ap[i] };
    double* o = out + 12 * (size_t)i;
#pragma unroll
    for (int k = 0; k < 6; k++) { o[2 * k] = w[k].x; o[2 * k + 1] = w[k].y; }
}

// staging layout: node state | rigid records | works | contact records, each 256-byte aligned
struct ckpt_layout { size_t nodes, rigid, works, cont, bytes; };
static ckpt_layout ckpt_sections(int nn, int nb, int ncont)
{
    auto up = [](size_t x) { return (x + 255) & ~(size_t)255; };
    ckpt_layout L;
    L.nodes = 0;
    L.rigid = up(sizeof(double) * 12 * (size_t)nn);
    L.works = L.rigid + up(sizeof(double) * MEL_RIGID_NF * (size_t)nb);
    L.cont = L.works + up(sizeof(double) * 7 * (size_t)nb);
    L.bytes = L.cont + up(sizeof(mel_contact) * (size_t)ncont) + 256;
    return L;
}

mel_status mel_checkpoint_start(mel_handle* h)
{
    if (!h) return MEL_ERR_INVALID;
    cudaSetDevice(h->device);
    mel_ckpt& k = h->ck;
    if (!k.side) {
        if (cudaStreamCreateWithFlags(&k.side, cudaStreamNonBlocking) != cudaSuccess ||
            cudaEventCreateWithFlags(&k.packed, cudaEventDisableTiming) != cudaSuccess ||
            cudaEventCreateWithFlags(&k.landed, cudaEventDisableTiming) != cudaSuccess) {
            mel_set_cuda_error(cudaGetLastError(), "checkpoint stream", __FILE__, __LINE__);
            return MEL_ERR_CUDA;
        }
    }
    // an unread snapshot is replaced; its copy must have landed before the staging is reused
    if (k.pending) MEL_CUDA_OK(cudaEventSynchronize(k.landed));
    k.pending = false;
    const ckpt_layout L = ckpt_sections(h->nn, h->nb, h->d.ncont);
    if (L.bytes > k.d_cap) {
        if (k.d_stage) cudaFree(k.d_stage);
        k.d_stage = nullptr; k.d_cap = 0;
        if (cudaMalloc(&k.d_stage, 2 * L.bytes) != cudaSuccess) { mel_set_error("checkpoint staging (device) allocation failed"); return MEL_ERR_OOM; }
        k.d_cap = 2 * L.bytes;
    }
    if (L.bytes > k.h_cap) {
        if (k.h_stage) cudaFreeHost(k.h_stage);
        k.h_stage = nullptr; k.h_cap = 0;
        if (cudaMallocHost(&k.h_stage, 2 * L.bytes) != cudaSuccess) { mel_set_error("checkpoint staging (pinned host) allocation failed"); return MEL_ERR_OOM; }
        k.h_cap = 2 * L.bytes;
    }
    // the snapshot is taken on the solver's stream, so it sees every step launched before this
    // call and none launched after it; only the device-to-host copy runs beside later steps
    if (h->nn > 0)
        ckpt_pack_nodes<<<(h->nn + 255) / 256, 256, 0, h->stream>>>(h->d.u, h->d.v, h->d.a, h->d.up, h->d.vp, h->d.ap,
                                                                     h->nn, reinterpret_cast<double*>(k.d_stage + L.nodes));
    MEL_CUDA_OK(cudaGetLastError());
    MEL_CUDA_OK(cudaMemcpyAsync(k.d_stage + L.rigid, h->d.rg, sizeof(double) * MEL_RIGID_NF * (size_t)h->nb, cudaMemcpyDeviceToDevice, h->stream));
    MEL_CUDA_OK(cudaMemcpyAsync(k.d_stage + L.works, h->d.works, sizeof(double) * 7 * (size_t)h->nb, cudaMemcpyDeviceToDevice, h->stream));
    if (h->d.ncont > 0)
        MEL_CUDA_OK(cudaMemcpyAsync(k.d_stage + L.cont, h->d.cont, sizeof(mel_contact) * (size_t)h->d.ncont, cudaMemcpyDeviceToDevice, h->stream));
    MEL_CUDA_OK(cudaEventRecord(k.packed, h->stream));
    // a batch member is stepped on the batch's stream: finish the snapshot before returning
    if (h->batch) MEL_CUDA_OK(cudaEventSynchronize(k.packed));
    MEL_CUDA_OK(cudaStreamWaitEvent(k.side, k.packed, 0));
    MEL_CUDA_OK(cudaMemcpyAsync(k.h_stage, k.d_stage, L.bytes, cudaMemcpyDeviceToHost, k.side));
    MEL_CUDA_OK(cudaEventRecord(k.landed, k.side));
    k.nn = h->nn; k.nb = h->nb; k.ncont = h->d.ncont;
    k.time = h->time; k.dt = h->dt; k.next_cup = h->next_cup;
    k.pending = true;
    return MEL_OK;
}

mel_status mel_checkpoint_read(mel_handle* h, double* node_state, double* rigid, double* works, mel_contact* contacts,
                               int contacts_capacity, int* ncont, double* time3)
{
    if (!h) return MEL_ERR_INVALID;
    mel_ckpt& k = h->ck;
    if (!k.pending) { mel_set_error("no checkpoint has been started since the last read"); return MEL_ERR_INVALID; }
    if (ncont) *ncont = k.ncont;
    if (contacts && contacts_capacity < k.ncont) {
        mel_set_error("checkpoint holds %d contact elements, the buffer %d", k.ncont, contacts_capacity);
        return MEL_ERR_INVALID;
    }
    cudaSetDevice(h->device);
    MEL_CUDA_OK(cudaEventSynchronize(k.landed));
    const ckpt_layout L = ckpt_sections(k.nn, k.nb, k.ncont);
    if (node_state) memcpy(node_state, k.h_stage + L.nodes, sizeof(double) * 12 * (size_t)k.nn);
    if (rigid) memcpy(rigid, k.h_stage + L.rigid, sizeof(double) * MEL_RIGID_NF * (size_t)k.nb);
    if (works) memcpy(works, k.h_stage + L.works, sizeof(double) * 7 * (size_t)k.nb);
    if (contacts && k.ncont > 0) memcpy(contacts, k.h_stage + L.cont, sizeof(mel_contact) * (size_t)k.ncont);
    if (time3) { time3[0] = k.time; time3[1] = k.dt; time3[2] = k.next_cup; }
    k.pending = false;
    return MEL_OK;
}

mel_status mel_get_time(mel_handle* h, double* time, double* dt)
{
    if (!h) return MEL_ERR_INVALID;
    if (time) *time = h->time;
    if (dt) *dt = h->dt;
    return MEL_OK;
}

mel_status mel_monitor_compute(mel_handle* h, mel_monitor* out)
{
    if (!h || !out) return MEL_ERR_INVALID;
    cudaSetDevice(h->device);
    memset(out, 0, sizeof *out);
    mel_launch_monitor(h->d, h->d_monitor_part, h->d_rigid_ids, h->nrigid, h->d_monitor, h->stream);
    double m[20];
    MEL_CUDA_OK(cudaMemcpyAsync(m, h->d_monitor, sizeof m, cudaMemcpyDeviceToHost, h->stream));
    MEL_CUDA_OK(cudaStreamSynchronize(h->stream));
    out->time = h->time;
    out->kinetic_energy = m[0];
    out->mean_displacement[0] = m[1];
    out->mean_displacement[1] = m[2];
    out->active_contacts = (int)m[3];
    out->n_contacts = h->d.ncont;
    for (int r = 0; r < h->nrigid && r < 4; r++) {
        out->rigid_force[2 * r] = m[4 + 4 * r]; out->rigid_force[2 * r + 1] = m[5 + 4 * r];
        out->rigid_dirichlet[2 * r] = m[6 + 4 * r]; out->rigid_dirichlet[2 * r + 1] = m[7 + 4 * r];
    }
    return MEL_OK;
}

const char* mel_last_error_string(void) { return g_err.c_str(); }
int mel_abi_version(void) { return MELGPU_ABI_VERSION; }

mel_status mel_get_kernel_times(mel_handle* h, double* ms_contact, double* ms_body, double* ms_rigid, double* ms_proximity, int* launches)
{
    if (!h) return MEL_ERR_INVALID;
    if (ms_contact) *ms_contact = h->t_contact;
    if (ms_body) *ms_body = h->t_body;
    if (ms_rigid) *ms_rigid = 0.;
    if (ms_proximity) *ms_proximity = h->t_prox;
    if (launches) *launches = h->launches;
    return MEL_OK;
}

mel_status mel_get_sizes(mel_handle* h, int* n_bodies, int* n_nodes, int* n_gauss, int* n_gp_entries, int* n_node_entries, int* n_border_nodes)
{
    if (!h) return MEL_ERR_INVALID;
    if (n_bodies) *n_bodies = h->nb;
    if (n_nodes) *n_nodes = h->nn;
    if (n_gauss) *n_gauss = h->ng;
    if (n_gp_entries) *n_gp_entries = h->nge;
    if (n_node_entries) *n_node_entries = h->nse;
    if (n_border_nodes) *n_border_nodes = h->ne;
    return MEL_OK;
}

mel_status mel_get_step_stats(mel_handle* h, double* ms_total, double* bytes_body, double* bytes_contact,
                              int* n_deformable_nodes, int* n_contacts)
{
    if (!h) return MEL_ERR_INVALID;
    if (ms_total) *ms_total = h->t_total;
    if (bytes_body) *bytes_body = h->bytes_body;
    if (bytes_contact) *bytes_contact = h->bytes_contact + (double)h->d.ncont * (2 * sizeof(mel_contact) + 8 + 5 * 16 * 2);
    if (n_deformable_nodes) *n_deformable_nodes = h->n_def_nodes;
    if (n_contacts) *n_contacts = h->d.ncont;
    return MEL_OK;
}

mel_status mel_get_kernel_config(mel_handle* h, int* chunk_cap, long long* body_smem, int* body_ctas)
{
    if (!h) return MEL_ERR_INVALID;
    if (chunk_cap) *chunk_cap = h->chunk_cap;
    if (body_smem) *body_smem = (long long)h->body_smem;
    if (body_ctas) *body_ctas = h->nblocks_body + h->nwide;
    return MEL_OK;
}

mel_status mel_get_error_words(mel_handle* h, unsigned* words, int n)
{
    if (!h || !words) return MEL_ERR_INVALID;
    unsigned w[MEL_E_NWORDS];
    MEL_CUDA_OK(cudaMemcpy(w, h->d.err, sizeof w, cudaMemcpyDeviceToHost));
    for (int i = 0; i < n && i < MEL_E_NWORDS; i++) words[i] = w[i];
    return MEL_OK;
}

} // extern "C"

// ---------------------------------------------------------------------------------------------
// batches: independent models advanced by shared launches
// ---------------------------------------------------------------------------------------------
struct mel_batch {
    int device = 0, precision = MEL_PREC_FP64;
    cudaStream_t stream = nullptr;
    std::vector<mel_handle*> members;
    std::vector<mel_dev> h_devs;         // member descriptors as last uploaded
    std::vector<int> h_thr0, h_cta0;     // prefix sums: contact-pass threads, body CTAs
    mel_dev* d_devs = nullptr;
    int* d_thr0 = nullptr;
    int* d_cta0 = nullptr;
    size_t cap = 0;                      // members the device arrays hold
    bool dirty = true;                   // descriptors changed (admission, retirement, proximity)
    size_t smem = 0;                     // largest body-kernel shared memory of the members
    size_t smem_small = 0;               // the same over the members that fit two CTAs per SM
    int nsmall = 0;                      // those members, ordered first
    size_t two_per_sm = 0;
    long long launches = 0;
    double ms_last = 0.;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    mel_prox_stage* pstage = nullptr;    // staging of the members' proximity runs
};

// Re-uploads the member descriptors and the work prefixes (the stream is idle afterwards).
static mel_status batch_refresh(mel_batch* b)
{
    const int n = (int)b->members.size();
    MEL_CUDA_OK(cudaStreamSynchronize(b->stream));
    if ((size_t)n > b->cap) {
        size_t cap = std::max((size_t)n, 2 * b->cap);
        cudaFree(b->d_devs); cudaFree(b->d_thr0); cudaFree(b->d_cta0);
        b->d_devs = nullptr; b->d_thr0 = nullptr; b->d_cta0 = nullptr;
        if (cudaMalloc(&b->d_devs, sizeof(mel_dev) * cap) != cudaSuccess ||
            cudaMalloc(&b->d_thr0, sizeof(int) * (cap + 1)) != cudaSuccess ||
            cudaMalloc(&b->d_cta0, sizeof(int) * (cap + 1)) != cudaSuccess) {
            mel_set_error("batch descriptor allocation failed");
            return MEL_ERR_OOM;
        }
        b->cap = cap;
    }
    if (!b->two_per_sm) {
        int smem_sm = 0, smem_res = 0;
        cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, b->device);
        cudaDeviceGetAttribute(&smem_res, cudaDevAttrReservedSharedMemoryPerBlock, b->device);
        b->two_per_sm = (size_t)(smem_sm / 2 - smem_res);
    }
    // members whose body kernel fits two CTAs per SM first: one launch of the body pass runs them
    // at that occupancy, a second the members that need more shared memory (one launch sized for
    // the largest member would hold every CTA to one per SM)
    std::stable_partition(b->members.begin(), b->members.end(),
                          [&](const mel_handle* h) { return h->body_smem <= b->two_per_sm; });
    b->h_devs.resize(n);
    b->h_thr0.assign(n + 1, 0);
    b->h_cta0.assign(n + 1, 0);
    b->smem = 0; b->smem_small = 0; b->nsmall = 0;
    for (int i = 0; i < n; i++) {
        mel_handle* h = b->members[i];
        b->h_devs[i] = h->d;
        b->h_thr0[i + 1] = b->h_thr0[i] + h->d.ncont + h->d.ne;
        b->h_cta0[i + 1] = b->h_cta0[i] + h->nblocks_body;
        b->smem = std::max(b->smem, h->body_smem);
        if (h->body_smem <= b->two_per_sm) { b->smem_small = std::max(b->smem_small, h->body_smem); b->nsmall = i + 1; }
    }
    if (n > 0) {
        MEL_CUDA_OK(cudaMemcpy(b->d_devs, b->h_devs.data(), sizeof(mel_dev) * n, cudaMemcpyHostToDevice));
        MEL_CUDA_OK(cudaMemcpy(b->d_thr0, b->h_thr0.data(), sizeof(int) * (n + 1), cudaMemcpyHostToDevice));
        MEL_CUDA_OK(cudaMemcpy(b->d_cta0, b->h_cta0.data(), sizeof(int) * (n + 1), cudaMemcpyHostToDevice));
    }
    b->dirty = false;
    return MEL_OK;
}

// Update_proximity of the members due at this step: one run of the pipeline serves all of them
// (one set of launches and two host read-backs on the batch stream, whatever their number).  A
// member whose positions diverged leaves the batch; the others go on.
static mel_status batch_proximity(mel_batch* b, const std::vector<mel_handle*>& due)
{
    std::vector<mel_prox_member> m(due.size());
    for (size_t i = 0; i < due.size(); i++) { m[i].d = &due[i]->d; m[i].P = &due[i]->P; }
    int launches = 0;
    const int rc = mel_run_proximity_many(m.data(), (int)m.size(), b->pstage, launches, b->stream);
    b->launches += launches;
    if (rc) return (mel_status)rc;
    for (size_t i = 0; i < due.size(); i++) {
        if (m[i].rc == MEL_ERR_NAN || m[i].rc == MEL_ERR_BOUNDS) {
            due[i]->failed = m[i].rc;
            due[i]->failed_msg = m[i].msg;
        } else if (m[i].rc) {
            mel_set_error("%s", m[i].msg.c_str());
            return (mel_status)m[i].rc;
        }
    }
    return MEL_OK;
}

// removes the members marked failed (their state stays as it was when they failed)
static void batch_drop_failed(mel_batch* b)
{
    for (size_t i = 0; i < b->members.size();) {
        mel_handle* h = b->members[i];
        if (h->failed) { b->members.erase(b->members.begin() + i); h->batch = nullptr; b->dirty = true; }
        else i++;
    }
}

mel_status mel_batch_create(int device, int precision, mel_batch** out)
{
    if (!out) { mel_set_error("null output"); return MEL_ERR_INVALID; }
    *out = nullptr;
    if (precision != MEL_PREC_FP64 && precision != MEL_PREC_MIXED) { mel_set_error("unknown precision %d", precision); return MEL_ERR_INVALID; }
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) { mel_set_error("no CUDA device"); return MEL_ERR_NO_DEVICE; }
    if (device < 0 || device >= ndev) { mel_set_error("device %d out of range", device); return MEL_ERR_INVALID; }
    mel_batch* b = new mel_batch();
    b->device = device;
    b->precision = precision;
    cudaSetDevice(device);
    if (cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreate(&b->e0) != cudaSuccess || cudaEventCreate(&b->e1) != cudaSuccess) {
        mel_set_cuda_error(cudaGetLastError(), "batch stream", __FILE__, __LINE__);
        delete b;
        return MEL_ERR_CUDA;
    }
    *out = b;
    return MEL_OK;
}

mel_status mel_batch_admit(mel_batch* b, mel_handle* h)
{
    if (h && h->solver != MEL_SOLVER_EULER) { mel_set_error("batches advance the Euler scheme; step Solver_step schemes with mel_step"); return MEL_ERR_UNSUPPORTED; }
    if (h && (h->d.fdamp || h->d.falid || h->n_deact || h->d.b_gscr)) {
        mel_set_error("models with damping matrices, ALID layers, DEACTIVATION entries or deformable bodies above %d nodes are stepped with mel_step, not in a batch", MEL_MAX_BODY_NODES);
        return MEL_ERR_UNSUPPORTED;
    }
    if (!b || !h) return MEL_ERR_INVALID;
    if (h->batch) { mel_set_error("the handle is already a member of a batch"); return MEL_ERR_INVALID; }
    if (h->device != b->device || h->precision != b->precision) {
        mel_set_error("the handle's device or precision differs from the batch's");
        return MEL_ERR_INVALID;
    }
    cudaSetDevice(b->device);
    MEL_CUDA_OK(cudaStreamSynchronize(h->stream));
    MEL_CUDA_OK(cudaStreamSynchronize(b->stream));
    if (h->parity == 1) {                        // a batch keeps each member's time in time2[0]
        MEL_CUDA_OK(cudaMemcpy(h->d.time2, h->d.time2 + 1, sizeof(double), cudaMemcpyDeviceToDevice));
        h->parity = 0;
    }
    h->batch = b;
    b->members.push_back(h);
    b->dirty = true;
    return MEL_OK;
}

mel_status mel_batch_retire(mel_batch* b, mel_handle* h)
{
    if (!b || !h || h->batch != b) { mel_set_error("the handle is not a member of this batch"); return MEL_ERR_INVALID; }
    cudaSetDevice(b->device);
    MEL_CUDA_OK(cudaStreamSynchronize(b->stream));
    b->members.erase(std::find(b->members.begin(), b->members.end(), h));
    h->batch = nullptr;
    b->dirty = true;
    return MEL_OK;
}

mel_status mel_batch_step(mel_batch* b, int nsteps, int run_proximity)
{
    if (!b || nsteps < 0) { mel_set_error("invalid arguments"); return MEL_ERR_INVALID; }
    cudaSetDevice(b->device);
    b->launches = 0;
    cudaEventRecord(b->e0, b->stream);
    for (int step = 0; step < nsteps; step++) {
        if (b->dirty) { mel_status rc = batch_refresh(b); if (rc) return rc; }
        const int n = (int)b->members.size();
        if (n == 0) break;
        mel_launch_batch_step(b->d_devs, b->d_thr0, b->h_thr0[n], b->d_cta0, b->h_cta0[b->nsmall], b->h_cta0[n], n,
                              b->precision == MEL_PREC_MIXED, b->smem_small, b->smem, b->stream);
        b->launches += 2 + (b->nsmall > 0) + (b->nsmall < n);
        cudaError_t le = cudaGetLastError();
        if (le != cudaSuccess) { mel_set_cuda_error(le, "batch step launch", __FILE__, __LINE__); return MEL_ERR_CUDA; }
        std::vector<mel_handle*> due;
        for (mel_handle* h : b->members) {
            h->time += h->dt;                                    // Code/Solver.h:86
            h->pressure_state = 1;
            if (run_proximity && h->time > h->next_cup - 1.e-6 * h->dt) {   // Code/main.cpp:191-196
                h->next_cup = h->next_cup + h->cup;
                due.push_back(h);
                if (h->d.record_forces) { mel_launch_contact_pressures(h->d, b->stream); b->launches += 3; h->pressure_state = 0; }
                else h->pressure_state = 2;
            }
        }
        if (!due.empty()) {
            mel_status rc = batch_proximity(b, due);
            if (rc) return rc;
            b->dirty = true;
            batch_drop_failed(b);
        }
    }
    cudaEventRecord(b->e1, b->stream);
    cudaError_t e = cudaStreamSynchronize(b->stream);
    if (e != cudaSuccess) { mel_set_cuda_error(e, "mel_batch_step", __FILE__, __LINE__); return MEL_ERR_CUDA; }
    float ms = 0.f;
    cudaEventElapsedTime(&ms, b->e0, b->e1);
    b->ms_last = ms;
    for (mel_handle* h : b->members) {
        mel_status rc = check_errors(h);
        if (rc == MEL_ERR_BOUNDS) { h->failed = rc; h->failed_msg = mel_last_error_string(); }
        else if (rc) return rc;
    }
    batch_drop_failed(b);
    return MEL_OK;
}

mel_status mel_get_health(mel_handle* h, int* failed)
{
    if (!h || !failed) return MEL_ERR_INVALID;
    *failed = h->failed;
    if (h->failed) mel_set_error("%s", h->failed_msg.c_str());
    return MEL_OK;
}

mel_status mel_batch_stats(mel_batch* b, double* ms_last_call, long long* launches, int* members)
{
    if (!b) return MEL_ERR_INVALID;
    if (ms_last_call) *ms_last_call = b->ms_last;
    if (launches) *launches = b->launches;
    if (members) *members = (int)b->members.size();
    return MEL_OK;
}

mel_status mel_batch_destroy(mel_batch* b)
{
    if (!b) return MEL_OK;
    cudaSetDevice(b->device);
    cudaStreamSynchronize(b->stream);
    for (mel_handle* h : b->members) h->batch = nullptr;
    cudaFree(b->d_devs); cudaFree(b->d_thr0); cudaFree(b->d_cta0);
    cudaEventDestroy(b->e0); cudaEventDestroy(b->e1);
    mel_prox_stage_free(b->pstage);
    cudaStreamDestroy(b->stream);
    delete b;
    return MEL_OK;
}
