// Internal definitions of the B200 solver: device-resident model and kernel entry points.
// Layout (HBM): body-sorted structure-of-arrays; node pairs (x,y) as double2 for 16-byte
// accesses; the Gauss points of a deformable body cut into chunks, each chunk one contiguous
// 16-byte-aligned image (header, dN/dx-dN/dy pairs, 16-bit body-local support indices, pull
// positions, per-point weights and offsets, touched-node records) that a single bulk copy
// moves into shared memory; contact elements in the reference's mel_contact record.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>
#include "melgpu.h"

#define MEL_BODY_THREADS 256      // threads per body CTA: point warps, pull warps, warp 7 (copies, contacts)
// The FP64 body kernel: warps 0-6 run each chunk's Gauss-point pass and then its pull, over two
// chunk buffers.  The mixed kernel: a pipeline of point warps, pull warps and a copy warp over a
// ring of three buffers.
#define MEL_STAGES(mx) ((mx) ? 3 : 2)     // chunk buffers
#define MEL_PT_WARPS_MX 4                 // point warps of the mixed pipeline (warps 4-6 pull)
#define MEL_CHUNK_GP_FP64 224     // Gauss points per chunk: one point thread each
#define MEL_CHUNK_GP_MX 128
#define MEL_PULL_WARPS 7          // warps 0-6 of the two-buffer loop: point pass, then pull
#define MEL_PIECE 8               // entries of one node a lane of the mixed pull sums before the warp combines
// mixed-precision bodies with at least this many support entries run the three-stage pipeline,
// the others the two-buffer loop.  Measured on B200 (mixed body pass): the pipeline takes 0.537 ms
// against 0.588 ms on the 2000-disc sample, but a 32-sample batch of the batched workload steps in
// 3.36 ms with it against 2.02 ms with the loop; so by default no body runs the pipeline
// (MELGPU_PIPE_MIN_ENTRIES, read by mel_create, sets another threshold)
#define MEL_PIPE_MIN_ENTRIES (1LL << 62)
#define MEL_BAR_BYTES 128         // the ring's mbarriers (3 per stage) and the abort flag
#define MEL_CHUNK_E_MAX 2048      // support entries per chunk, upper bound (the host may choose less)
#define MEL_CHUNK_E_MAX_MX 3584   // the same for the mixed pass's FP32 images (its caps above 2048 come from the tuning table)
#define MEL_WAIT_NS 1000000000ull // bound of every device-side wait (1 s)
#define MEL_NBR_CAP_DEFAULT 64    // neighbour slots per body (grown on overflow)
#define MEL_MAX_BODY_NODES 4096   // nodes per deformable body held in shared memory
#define MEL_MAX_WIDE_NODES 65535  // larger bodies keep their node arrays in global memory (16-bit indices)
// bytes of a wide body's node arrays in global memory (mel_dev::gscr): s_f, s_fc, s_upf, then the
// post-loop arrays s_fn, s_fd, s_vp, s_ap, the six work terms and the temporary parameters
__host__ __device__ inline long long mel_wide_pre_bytes(int n) { return 32LL * n + 8LL * ((n + 1) & ~1); }
__host__ __device__ inline long long mel_wide_bytes(int n) { return mel_wide_pre_bytes(n) + (64LL + 48LL + 16LL) * n; }
#define MEL_SEGB 16               // segments per segment-block box (proximity pruning)
#define MEL_SEGB2 16              // blocks per superblock box (second pruning level)
#define MEL_MAX_SHIFT_SPAN 64     // periods one border box may span at a proximity update

// device error words (mel_dev::err)
enum { MEL_E_BOUNDS = 0, MEL_E_NBR_OVERFLOW = 1, MEL_E_STALE = 2, MEL_E_NAN = 3, MEL_E_CAPACITY = 4,
       MEL_E_NBR_NEED = 5, MEL_E_WAIT = 6, MEL_E_PRESSURE = 7, MEL_E_DEACT = 8, MEL_E_NWORDS = 9 };
#define MEL_PRESSURE_CAP 64       // contact contributions one border entry's pressure gathers

// Chunk image (all offsets in bytes from the image start, every section 16-byte aligned):
//   header   int4 {ngp, ne, ntn, nroff}
//   dN       ne x double2          dN/dx, dN/dy of every stored entry (float2 in the images of
//                                  the mixed-precision pass)
//   idx      ne x uint16           body-local support node of each entry
//   tpos     ne x uint16           entry positions in pull order, in pull rows (below)
//   c0       ngp2 x double         weight x jacobian of each point slot (ngp2 = ngp rounded to 2)
//   gpm      ngp4 x uint32         point slot: row table start | lane << 10 | support count << 15
//   tn       tn4 x uint32          pull slot: node | entry count << 12 | row table start << 20
//   tnode    ntn8 x uint16         (wide bodies only) each pull slot's node, 16 bits
//   roff     nroff8 x uint16       row tables: the point groups' rows, then the pull groups'
//                                  rows; each value is an offset (12 bits) | lane swizzle << 12
// Point slots: the chunk's points sorted by (support count descending, index), cut into groups of
// up to 32 slots, one warp each.  Row k of a group holds entry k of every slot whose point has
// more than k supports; these slots are a prefix of the group, so entry k of lane j sits at
// (r & 0xfff) + (j ^ (r >> 12)) with r = roff[r0 + k]: the lanes of a warp touch a permutation of
// consecutive entries.  The swizzle (k & 7 in rows whose width is a multiple of 8, else 0) spreads
// the entries of one point over the shared-memory bank groups.
// Pull slots: the touched nodes sorted by entry count (descending), cut into groups of 32 (slot t
// is lane t & 31 of group t >> 5).  Row j of a pull group holds, for every slot with more than j
// entries, the position of its node's entry j; a node's entries are in ascending point order.
// ne is the number of entries rounded up to a multiple of 8 (zero entries at the end).
// Images of the mixed pass's two-buffer loop replace the pull slots by pieces: tpos lists the
// positions of all entries in (node, point) order; the tn section holds MEL_PULL_WARPS + 1 uint16
// warp bounds (16 bytes), then one uint32 record per piece (first listed entry | (count - 1) << 13 |
// node << 16, 16 bits of node), a piece being at most MEL_PIECE consecutive entries of one node.  Pull warp w takes
// the pieces [bound w, bound w+1), which start and end at node boundaries; nroff counts the point
// rows only.
struct mel_chunk {        // one chunk of a body's Gauss points
    long long img;        // byte offset of the image in mel_dev::img
    int bytes;            // image size (multiple of 16)
    int ngp, ne, ntn;
    int gp0;              // first Gauss point (global index)
    int pad;
};

struct mel_chunk_layout {  // section offsets of an image
    int dN, idx, tpos, c0, gpm, tn, tnode, roff, bytes;
};
// dnb: bytes of one dN pair, 16 (FP64 images) or 8 (FP32 images of the mixed-precision pass).
// wide: the FP64 image of a body above MEL_MAX_BODY_NODES nodes, whose pull slots take their
// node from a uint16 section tnode (ntn8 entries) after tn instead of the record's 12 bits
__host__ __device__ inline mel_chunk_layout mel_chunk_sections(int ngp, int ne, int ntn, int nroff, int dnb, int wide = 0)
{
    mel_chunk_layout L;
    L.dN = 16;
    L.idx = L.dN + dnb * ne;
    L.tpos = L.idx + 2 * ne;
    L.c0 = L.tpos + 2 * ne;
    L.gpm = L.c0 + 8 * ((ngp + 1) & ~1);
    L.tn = L.gpm + 4 * ((ngp + 3) & ~3);
    L.tnode = L.tn + 4 * ((ntn + 3) & ~3);
    L.roff = L.tnode + (wide ? 2 * ((ntn + 7) & ~7) : 0);
    L.bytes = L.roff + 2 * ((nroff + 7) & ~7);
    return L;
}

struct mel_dev {
    // sizes
    int nb, nn, nbd, ne, ng, nchunk, ncont, cont_cap;
    int nmat, self_contact, record_forces, precision;
    double xmin, period, gx, gy;
    // time: time2[parity] is the step's start time, time2[parity^1] its end (ping-pong)
    double* time2;
    double* dt;
    // materials and laws
    const int* mat_type; const double* mat_p;
    const int* law_type; const int* law_len; const double* law_p; const int* table;
    // bodies
    const int *b_type, *b_mat, *b_per, *b_node0, *b_bd0, *b_chunk0, *b_order;
    int* b_status;           // MEL_STATUS_*; Update_status turns bodies inactive during the run
    double* b_damage;        // Body::damage: the running value of Update_damage (starts at 0)
    const double* b_dist;
    const int* b_has_bc;     // body has a non-"none" border condition
    // bodies above MEL_MAX_BODY_NODES nodes: byte offset of the body's node arrays in gscr (-1 for
    // the others, whose node arrays live in shared memory); NULL when the model has none
    const long long* b_gscr;
    char* gscr;
    double *rg, *rf, *rtot, *drv, *works;
    // nodes
    const double2 *X0, *minv, *mass;
    double2 *x, *u, *v, *a, *up, *vp, *ap;
    const int* sup_ptr; const uint16_t* sup_idx; const double* sup_N;
    // the same supports of deformable bodies laid out for the kinematics: a body's nodes as slots
    // sorted by support count (slot ranges start at multiples of 32), groups of 32 slots; slot
    // record = node | support count << 16; entry k of lane l of group G at kg_base[G] + 32 k + l
    const int* b_ks0; const unsigned* ks_rec; const int* kg_base;
    const uint16_t* ks_idx; const double* ks_N;
    double2 *o_fint, *o_fcon, *o_fneu, *o_fdir, *o_ftot;
    // damping matrices (Body::Update_damping_forces): for each degree of freedom (2 node + direction)
    // the terms it receives, in matrix-entry order: source degree of freedom and coefficient; the
    // damping forces of the step (NULL without matrices)
    const int *dmp_ptr, *dmp_src;
    const double* dmp_c;
    double2* fdamp;
    // ALID layers (Body::Update_alid_forces): the bodies with a layer, each body's x and y history of
    // the layer's reference velocity, alid_beta per node, and per receiving degree of freedom its
    // stiffness terms (source degree of freedom, k / (1/alpha0 + 1/alpha1)) in entry order
    int n_alid;
    const int *alid_b, *alid_hptr;
    const double *alid_ht, *alid_hv, *alid_beta;
    const int *al_ptr, *al_src;
    const double* al_c;
    double2* falid;
    // borders and border entries
    const int *bd_body, *bd_per, *bd_bef, *bd_aft, *bd_e0, *bd_bc, *bd_h0;
    const double *bd_bcp, *ht, *hv;
    const int *e_node, *e_sn, *e_ss;         // e_sn/e_ss: 4 per entry (node0..3, shift0..3)
    const double* e_len0;
    double* e_len;                            // lengths of the last Update_borders
    double2* e_bcp;                           // border-condition pressures of the last Update_bc_forces
                                              // (Border::x_bc_pressure, y_bc_pressure; zero on borders
                                              // whose conditions are both none)
    int nblk;                                 // segment blocks (MEL_SEGB segments of one border)
    const int* bd_blk0;                       // [nbd+1] first block of each border
    const int* blk_border;                    // border of each block
    double4* seg_blk;                         // block boxes of the current proximity update
    int nsblk;                                // superblocks (MEL_SEGB2 consecutive blocks of one border)
    const int* bd_sblk0;                      // [nbd+1] first superblock of each border
    const int* sblk_border;                   // border of each superblock
    double4* seg_sblk;                        // superblock boxes (unions of their block boxes)
    // Gauss points: chunk table and chunk images
    const mel_chunk* chunk;
    const int* b_pipe;                        // per body: 1 = three-stage pipeline (mixed pass), else
                                              // the two-buffer loop; NULL for FP64
    const char* img;
    int img_cap;                              // bytes of one shared-memory staging buffer
    // contacts
    mel_contact* cont;
    double* cont_w;                           // per-contact work increment of the last law evaluation
    double* cont_rt;                          // 6 per contact: rigid slave and rigid master force and
                                              // moment terms of the last contact pass (arms from the
                                              // positions before the body kernel moves any node)
    int any_damped;                           // a law with work terms is in use
    const int* b_cont0;                       // [nb+1] slave contact ranges (list is body-major)
    const int* b_inc0;                        // [nb+1] into inc_rng
    const int2* inc_rng;                      // incoming (master-side) contact ranges in send order
    // Solver_step (Code/Solver.h:98-486): phase of an adaptive launch (1: first half-step, 2: second
    // half-step), scheme and its parameters (mel_model_desc::solver_params), inverse distance
    // estimators of the nodes (Code/IO.h:1620,1819), temporary displacement parameters and
    // displacements, nodal errors, nodal mass-scaling factors; per body: total and largest error,
    // scaled mass, rigid mass-scaling factor and its last increment, rigid temporary kinematics
    // (x, y, r displacement then velocity)
    int phase, solver;
    double sp[8];
    const double* ide;
    double2 *upt, *ut, *errv, *fms;
    double *terr, *merr, *bmms, *bfms, *bdfms, *rg_tmp;
    // border contact pressures (Update_contact_pressures): per border entry, the contributions
    // gathered (contact << 2 | role, at most MEL_PRESSURE_CAP) and the pressures
    int* cp_cnt; int* cp_item;
    double *cpx, *cpy;
    // bound of the body kernel's pipeline waits (MEL_WAIT_NS; the environment variable
    // MELGPU_WAIT_NS read by mel_create shortens it so that tests can make a wait give up)
    unsigned long long wait_ns;
    // error words
    unsigned int* err;
};

// kernel launch wrappers (mel_kernels.cu)
// Update_damping_forces of every deformable body with matrices, from the velocity parameters
void mel_launch_damping(const mel_dev& d, cudaStream_t s);
// Update_alid_forces at the step's start time time2[parity], or at T when use_T (Solver_step)
void mel_launch_alid(const mel_dev& d, int parity, double T, int use_T, cudaStream_t s);
void mel_launch_contact(const mel_dev& d, double law_dt_scale, cudaStream_t s);
// Initialize_CZM's pass over the contact list (contact geometry, then the initial bonds)
void mel_launch_czm_init(const mel_dev& d, cudaStream_t s);
// nblocks: bodies b_order[0, nblocks); nwide: the wide bodies after them
void mel_launch_body(const mel_dev& d, int parity, int nblocks, size_t smem, cudaStream_t s, int nwide = 0);
// one half-step of Solver_step (d.phase 1 or 2): T0 = Time, Tf = the time the forces see
void mel_launch_body_adaptive(const mel_dev& d, double T0, double Tf, int nblocks, size_t smem, cudaStream_t s, int nwide = 0);
// Solver_step's error and mass sums over the bodies in order (Code/Solver.h:289-331): out =
// {mean_error, max_error, total_mass, max_mass}
void mel_launch_error_reduce(const mel_dev& d, double* out, cudaStream_t s);
// Update_bc(T) of every body's driven degrees of freedom (mel_dev::drv)
void mel_launch_drivendof(const mel_dev& d, double T, cudaStream_t s);
// Body::Restore of the rigid bodies' kinematics from a copy of the rigid records
void mel_launch_rigid_restore(const mel_dev& d, const double* rg_snap, cudaStream_t s);
// one step of a batch: the contact pass over thr0[nsamp] threads, the body pass over cta0[nsamp]
// CTAs and the per-sample time advance (devs, thr0, cta0 in device memory).  The body pass is two
// launches: CTAs [0, ncta_small) with smem_small bytes (members whose bodies fit two CTAs per SM,
// ordered first), then the rest with smem bytes
void mel_launch_batch_step(const mel_dev* devs, const int* thr0, int nthr, const int* cta0, int ncta_small, int ncta,
                           int nsamp, int mixed, size_t smem_small, size_t smem, cudaStream_t s);
size_t mel_body_smem_bytes(int max_nodes, int max_image_bytes, int mixed, int stages);
void mel_launch_update_borders(const mel_dev& d, cudaStream_t s);
void mel_launch_monitor(const mel_dev& d, double* part, const int* rigid_ids, int nrigid, double* out, cudaStream_t s);
// Update_contact_pressures (Code/Proximity.h:1014-1069) from the current contact list
void mel_launch_contact_pressures(const mel_dev& d, cudaStream_t s);

// one monitored entry of STATIC_CONTROL's MONITORING list (the vector Read_spy_line builds,
// Code/IO.h:11-590): type (0 position, 1 displacement, 2 velocity, 3 acceleration, 4 force,
// 7 contact, 9 energy, 10 work), kind (component or quantity), sub (force kind), body, node (-1:
// the whole body), border and border node (contact entries)
struct mel_mon_op { int type, kind, sub, body, node, border, bnode, pad; };
// the row's leading columns (Code/Monitoring.h:25)
struct mel_mon_head { double iteration, time, dt, neval, max_error, mean_error; };
// Monitoring after a step: per-body partial sums into part[3*nb], then the row into row[0..]
// (row[0] = number of values that follow)
// Update_status (Code/Proximity.h:550-1007): the DEACTIVATION entries (MEL_DEACT_NF doubles each)
// evaluated on the current state; bodies whose condition holds become inactive
void mel_launch_status(const mel_dev& d, const double* entries, int n, cudaStream_t s);
void mel_launch_monitor(const mel_dev& d, const mel_mon_op* ops, int nops, int energy, int boundaries,
                        double* part, double* row, const mel_mon_head& hd, cudaStream_t s);

int mel_body_kernel_configure(size_t smem);

#define MEL_CUDA_OK(call) do { cudaError_t e_ = (call); if (e_ != cudaSuccess) { mel_set_cuda_error(e_, #call, __FILE__, __LINE__); return MEL_ERR_CUDA; } } while (0)
void mel_set_cuda_error(cudaError_t e, const char* what, const char* file, int line);
void mel_set_error(const char* fmt, ...);
