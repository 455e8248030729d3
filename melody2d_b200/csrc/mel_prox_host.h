// Host-side state of the proximity pipeline (mel_prox.cu) owned by a solver handle.
#pragma once
#include <vector>
#include "mel_internal.h"

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
    int2* inc_rng = nullptr; size_t inc_rng_bytes = 0;
    int* b_inc0 = nullptr; int* b_cont0 = nullptr;
    int* e_cnt = nullptr; int* e_ptr = nullptr; int* e_cur = nullptr;
    int* e_list = nullptr; size_t e_list_bytes = 0;
    size_t cont_bytes = 0;
    mel_contact* cont_alt = nullptr; size_t cont_alt_bytes = 0;
    double* cont_w = nullptr; size_t cont_w_bytes = 0;
    double* cont_rt = nullptr; size_t cont_rt_bytes = 0;
    int* scan_ws = nullptr; size_t scan_ws_bytes = 0;    // scan block totals
    int ntask = 0, nslot = 0;
    int launches = 0;                                      // kernels launched by the pipeline (running count)
};

struct mel_prox_host {
    std::vector<int> b_type, b_per, b_bd0, bd_e0;
};

int mel_run_proximity(mel_dev& d, mel_prox_state& P, const mel_prox_host& H, cudaStream_t s);
int mel_index_contacts(mel_dev& d, mel_prox_state& P, cudaStream_t s);
int mel_index_external(mel_dev& d, mel_prox_state& P, const mel_contact* host_list, int n, cudaStream_t s);
int mel_scan_exclusive(const int* in, int* out, int n, mel_prox_state& P, cudaStream_t s);
