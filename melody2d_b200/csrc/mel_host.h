// Host model read from the reference's input files (STATIC_CONTROL.asc, STATIC_DATA.asc,
// DYNAMIC_nnnnn.asc) and exposed as a mel_model_desc.
#pragma once
#include <string>
#include <vector>
#include "melgpu.h"

struct mel_host_model {
    mel_model_desc desc;
    std::string name;
    std::vector<int> material_type, law_type, law_length, contacts_table;
    std::vector<double> material_params, law_params;
    std::vector<std::string> material_names;
    std::vector<int> body_type, body_material, body_periodic, body_status, body_node_ptr, body_border_ptr, body_gp_ptr,
        body_cell_ptr, n_regions;
    std::vector<double> body_dist, rigid;
    std::vector<double> node_x0, node_mass, node_inv_mass, node_domain, node_sup_N, node_state;
    std::vector<int> node_sup_ptr, node_sup_idx;
    std::vector<int> border_body, border_periodicity, border_interpolant, border_before, border_after, border_node_ptr,
        border_nodes, border_bc_type, border_hist_ptr;
    std::vector<double> border_bc_param, hist_time, hist_value;
    std::vector<int> gp_sup_ptr, gp_sup_idx;
    std::vector<double> gp_N, gp_dNdx, gp_dNdy, gp_weight, gp_jacobian;
    std::vector<int> cells, body_matrix_ptr, matrix_dofs;
    std::vector<double> matrix_stiffness, matrix_damping;
    std::vector<int> body_alid_ptr;                       // empty: no ALID layer
    std::vector<double> alid_time, alid_value, node_alid;
    std::vector<mel_contact> contacts;   // CONTACTS of the DYNAMIC file
    // run control that drives output only: Save_period, Print_period (STATIC_CONTROL SOLVER block),
    // Number_save, Number_iteration, Number_print, Next_save, Next_print (DYNAMIC SOLVER block), and
    // the MONITORING entries as Read_spy_line builds them (Code/IO.h:933-945)
    double save_period = 0., print_period = 0., next_save = 0., next_print = 0.;
    int number_save = 0, number_iteration = 0, number_print = 0;
    std::vector<std::vector<double>> monitored;
    // DEACTIVATION entries (Code/IO.h:947-968), and the same zero-padded for mel_model_desc
    std::vector<std::vector<double>> deactivated;
    std::vector<double> deactivated_flat;
    void finalize();                     // points desc at the vectors
};

mel_status mel_load_files(const char* dir, int restart_index, mel_host_model* out);

extern "C" {
// extra entry points (declared here for C++ callers; see include/melgpu.h for the main ABI)
mel_status mel_set_rigid(mel_handle* h, const double* rigid);
mel_status mel_set_time(mel_handle* h, double time, double dt, double next_contact_update);
mel_status mel_record_forces(mel_handle* h, int on);
mel_status mel_set_timing(mel_handle* h, int on);
mel_status mel_get_error_words(mel_handle* h, unsigned* words, int n);
}
