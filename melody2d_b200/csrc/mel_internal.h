// Internal definitions of the B200 solver: device-resident model and kernel entry points.
// Layout (HBM): body-sorted structure-of-arrays; node pairs (x,y) as double2 for 16-byte
// accesses; Gauss-point supports stored per chunk (<= MEL_CHUNK_GP points, <= MEL_CHUNK_E
// entries, start padded to 8 entries so every chunk begins on a 16-byte boundary) with
// 16-bit body-local indices; contact elements in the reference's mel_contact record.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>
#include "melgpu.h"

#define MEL_CHUNK_GP 128          // Gauss points per chunk (one thread each in the forward pass)
#define MEL_CHUNK_E 2048          // support entries per chunk (shared-memory staging capacity)
#define MEL_BODY_THREADS 256      // threads per body CTA
#define MEL_NBR_CAP_DEFAULT 64    // neighbour slots per body (grown on overflow)
#define MEL_MAX_BODY_NODES 4096   // nodes per deformable body held in shared memory

// device error words (mel_dev::err)
enum { MEL_E_BOUNDS = 0, MEL_E_NBR_OVERFLOW = 1, MEL_E_STALE = 2, MEL_E_NAN = 3, MEL_E_CAPACITY = 4,
       MEL_E_NBR_NEED = 5, MEL_E_NWORDS = 8 };

struct mel_chunk {        // one chunk of a body's Gauss points
    int gp0;              // first Gauss point (global index)
    int ngp;              // Gauss points in the chunk
    int e0;               // first entry (padded global entry index, multiple of 8)
    int ne;               // entries (padded to a multiple of 8)
    int tn0;              // first touched-node record
    int ntn;              // touched nodes
    int pad0, pad1;
};

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
    const int *b_type, *b_mat, *b_per, *b_status, *b_node0, *b_bd0, *b_chunk0, *b_order;
    const double* b_dist;
    const int* b_has_bc;     // body has a non-"none" border condition
    double *rg, *rf, *rtot, *drv, *works;
    // nodes
    const double2 *X0, *minv, *mass;
    double2 *x, *u, *v, *a, *up, *vp, *ap;
    const int* sup_ptr; const uint16_t* sup_idx; const double* sup_N;
    double2 *o_fint, *o_fcon, *o_fneu, *o_fdir, *o_ftot;
    // borders and border entries
    const int *bd_body, *bd_per, *bd_bef, *bd_aft, *bd_e0, *bd_bc, *bd_h0;
    const double *bd_bcp, *ht, *hv;
    const int *e_node, *e_sn, *e_ss;         // e_sn/e_ss: 4 per entry (node0..3, shift0..3)
    const double* e_len0;
    double* e_len;                            // lengths of the last Update_borders
    // Gauss points
    const double* gp_c0; const int* gp_e0; const uint8_t* gp_ns;
    const uint16_t *ge_idx, *ge_tpos; const double2* ge_dN;
    const float2* ge_dNf;                     // FP32 copy for the mixed-precision pass
    const mel_chunk* chunk;
    const uint16_t *tn_node, *tn_start, *tn_cnt;
    // contacts
    mel_contact* cont;
    double* cont_w;                           // per-contact work increment of the last law evaluation
    int any_damped;                           // a law with work terms is in use
    const int* b_cont0;                       // [nb+1] slave contact ranges (list is body-major)
    const int* b_inc0;                        // [nb+1] into inc_rng
    const int2* inc_rng;                      // incoming (master-side) contact ranges in send order
    // error words
    unsigned int* err;
};

// kernel launch wrappers (mel_kernels.cu)
void mel_launch_contact(const mel_dev& d, double law_dt_scale, cudaStream_t s);
void mel_launch_body(const mel_dev& d, int parity, int nblocks, size_t smem, cudaStream_t s);
size_t mel_body_smem_bytes(int max_nodes, int max_border_nodes);
void mel_launch_update_borders(const mel_dev& d, cudaStream_t s);
void mel_launch_monitor(const mel_dev& d, double* part, const int* rigid_ids, int nrigid, double* out, cudaStream_t s);

void mel_body_kernel_configure(size_t smem);
// proximity (mel_prox.cu)
void mel_scan_exclusive(const int* in, int* out, int n, cudaStream_t s);

#define MEL_CUDA_OK(call) do { cudaError_t e_ = (call); if (e_ != cudaSuccess) { mel_set_cuda_error(e_, #call, __FILE__, __LINE__); return MEL_ERR_CUDA; } } while (0)
void mel_set_cuda_error(cudaError_t e, const char* what, const char* file, int line);
void mel_set_error(const char* fmt, ...);
