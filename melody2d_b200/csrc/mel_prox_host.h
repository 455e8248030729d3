// Host-side state of the proximity pipeline (mel_prox.cu) owned by a solver handle, and the job
// table through which one set of launches serves several models (the members of a batch).
#pragma once
#include <string>
#include <vector>
#include "mel_internal.h"

struct mel_prox_stage;   // staging buffers of a run (pinned host + device), opaque

struct mel_prox_state {
    int nbr_cap = MEL_NBR_CAP_DEFAULT;
    int* nbr = nullptr; int* nbn = nullptr;
    double* aabb = nullptr; int* shmin = nullptr; int* shmax = nullptr;
    void* task = nullptr; size_t task_bytes = 0;            // int4 per task
    int* tns = nullptr; size_t tns_bytes = 0;               // slave border nodes per task
    int* tslot = nullptr; size_t tslot_bytes = 0;           // first slot of each task
    int* tkey = nullptr; size_t tkey_bytes = 0;             // master body of each task
    int* tcnt = nullptr; int* btask0 = nullptr;             // per body: task count, first task
    int* scnt = nullptr; int* bslot0 = nullptr;             // per body: slot count, first slot
    int* inc_task = nullptr; size_t inc_task_bytes = 0;
    int* slot_cnt = nullptr; size_t slot_bytes = 0;
    int* slot_off = nullptr; size_t slot_off_bytes = 0;
    int* tmap = nullptr; size_t tmap_bytes = 0;             // task of each slot
    int* nzoff = nullptr; size_t nzoff_bytes = 0;           // slots with candidates: offsets, list
    int* nzlist = nullptr; size_t nzlist_bytes = 0;
    int nnz = 0;
    int2* inc_rng = nullptr; size_t inc_rng_bytes = 0;
    int* b_inc0 = nullptr; int* b_cont0 = nullptr;
    int* e_cnt = nullptr; int* e_ptr = nullptr; int* e_cur = nullptr;
    int* e_list = nullptr; size_t e_list_bytes = 0;
    size_t cont_bytes = 0;
    mel_contact* cont_alt = nullptr; size_t cont_alt_bytes = 0;
    double* cont_w = nullptr; size_t cont_w_bytes = 0;
    double* cont_rt = nullptr; size_t cont_rt_bytes = 0;
    int* scan_ws = nullptr; size_t scan_ws_bytes = 0;    // scan block totals
    // cell-list broad phase (cl_on): bucket counts / cursors and starts (cl_T + 1 each), border
    // indices by bucket, the run's largest box width and height; cell side cl_h, columns cl_hx
    // (cl_ncx per period)
    int cl_on = 0, cl_T = 0, cl_ncx = 1;
    double cl_h = 0., cl_hx = 0.;
    int *cl_cnt = nullptr, *cl_cur = nullptr, *cl_start = nullptr, *cl_idx = nullptr;
    unsigned long long* cl_w = nullptr;
    int ntask = 0, nslot = 0;
    int launches = 0;                                      // kernels launched by the pipeline (running count)
    mel_prox_stage* stage = nullptr;                       // staging of this handle's own runs
};

struct mel_prox_host {
    std::vector<int> b_type, b_per, b_bd0, bd_e0;
};

// One model's part of a run, as the kernels see it: its descriptor and its own buffers.
struct mel_prox_job {
    mel_dev d;
    double* aabb; int* shmin; int* shmax;
    int* nbr; int* nbn; int nbr_cap;
    int ntask, nslot, have_old;
    int4* task; int* tns; int* tslot; int* tkey;
    int* tcnt; int* btask0; int* scnt; int* bslot0;
    int* slot_cnt; int* slot_off; int* inc_task; int* tmap;
    int* nzoff; int* nzlist; int nnz;
    int2* inc_rng; int* b_inc0; int* b_cont0;
    int* e_cnt; int* e_ptr; int* e_cur; int* e_list;
    mel_contact* cont_new;        // the list being written (write stage)
    int* readback;                // this member's words of the run's read-back array
    int cl_on, cl_T, cl_ncx;      // cell-list broad phase (mel_prox_state)
    double cl_h, cl_hx;
    int *cl_cnt, *cl_cur, *cl_start, *cl_idx;
    unsigned long long* cl_w;
};

// A model taking part in a run.  rc: MEL_OK, or the member's own failure (MEL_ERR_NAN,
// MEL_ERR_BOUNDS) with msg; the other members carry on.
struct mel_prox_member {
    mel_dev* d;
    mel_prox_state* P;
    int rc = 0;
    std::string msg;
};

// Update_proximity of several models with one set of launches on stream s.  Returns MEL_OK when
// the run itself went through (members may still have failed: see their rc), else the status of
// a failure that stops every member (allocation, CUDA).  launches: kernels launched.
int mel_run_proximity_many(mel_prox_member* m, int n, mel_prox_stage*& stage, int& launches, cudaStream_t s);
void mel_prox_stage_free(mel_prox_stage* stage);

int mel_run_proximity(mel_dev& d, mel_prox_state& P, const mel_prox_host& H, cudaStream_t s);
int mel_index_external(mel_dev& d, mel_prox_state& P, const mel_contact* host_list, int n, cudaStream_t s);
