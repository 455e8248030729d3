// melody_gpu: host main of the B200 solver, the loop of the reference's Code/main.cpp:25-239 with the
// solver, Monitoring and the proximity cadence on the GPU through include/melgpu.h.
//
//   melody_gpu <restart_index> [case_dir] [max_steps_per_call]
//
// Reads STATIC_CONTROL.asc / STATIC_DATA.asc / DYNAMIC_<restart>.asc from case_dir (default: the
// current directory, as the reference), runs the set-up (Code/main.cpp:104-127) and the time loop
// until Tend.  Per iteration (Code/main.cpp:141-238): the solver step, Monitoring (unless
// NO_MONITORING; rows stay on the device until the save), the proximity update when due, the print
// counter (Write_graphic itself is graphics output and is not produced), and at each save
// Write_dynamic (DYNAMIC_nnnnn.asc) and Write_monitoring (rows appended to MONITORING.asc), both in
// the reference's layout and number formatting.  Steps between events are batched into one
// mel_step call: under the Euler scheme the host repeats the loop's Time += Deltat to find the
// iteration at which the next save or print falls; the adaptive schemes step one iteration per
// call.  Exit status is non-zero on any solver error, including non-finite state.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <iomanip>
#include <string>
#include <vector>
#include "melgpu.h"

static int fail(const char* what, mel_status rc)
{
    std::fprintf(stderr, "%s failed (%d): %s\n", what, (int)rc, mel_last_error_string());
    return rc ? (int)rc : 1;
}

int main(int argc, char** argv)
{
    if (argc < 2) {
        std::fprintf(stderr, "usage: %s restart_index [case_dir] [max_steps_per_call]\n", argv[0]);
        return 2;
    }
    const int restart = std::atoi(argv[1]);
    const std::string dir = argc > 2 ? argv[2] : ".";
    int chunk = argc > 3 ? std::atoi(argv[3]) : 1000;
    if (chunk < 1) chunk = 1;

    mel_model_desc* desc = nullptr;
    void* owner = nullptr;
    mel_status rc = mel_load_desc(dir.c_str(), restart, &desc, &owner);
    if (rc) return fail("mel_load_desc", rc);
    static mel_run_control run;
    if ((rc = mel_load_run_control(owner, &run))) { mel_free_desc(owner); return fail("mel_load_run_control", rc); }
    const double tend = desc->tend;
    const bool euler = desc->solver == MEL_SOLVER_EULER;
    const bool monitoring = run.flags[8] == 0;                 // NO_MONITORING (Code/main.cpp:173)
    mel_options opt = { MEL_PREC_FP64, 0, 0, 0 };
    mel_handle* h = nullptr;
    rc = mel_create_loaded(owner, &opt, &h);
    mel_free_desc(owner);
    if (rc) return fail("mel_create_loaded", rc);

    int row_len = 0;
    if (monitoring) {
        rc = mel_monitor_setup(h, run.monitored, run.n_monitored, run.flags[1], run.flags[2], chunk,
                               run.number_iteration, &row_len);
        if (rc) { mel_destroy(h); return fail("mel_monitor_setup", rc); }
    }
    std::vector<double> rows, held;                 // held: rows since the last save, as the reference keeps them
    if (monitoring) rows.resize((size_t)chunk * (row_len + 1));

    int number_save = run.number_save, number_print = run.number_print, number_iteration = run.number_iteration;
    double next_save = run.next_save, next_print = run.next_print;
    double time = 0., dt = 0.;
    mel_get_time(h, &time, &dt);
    while (time < tend) {
        // iterations until the next save, print or the end, repeating Time += Deltat on the host
        int k = 1;
        bool save_due = false;
        if (euler) {
            double t = time;
            for (k = 1; k <= chunk; k++) {
                t = t + dt;
                if (t > next_save - 1.e-6 * dt) { save_due = true; break; }
                if (t > next_print - 1.e-6 * dt || !(t < tend)) break;
            }
            if (k > chunk) k = chunk;
        }
        mel_step_io io = {};
        if (k > 1) {
            io.nsteps = k - 1;
            io.run_proximity = 1;
            if ((rc = mel_step(h, &io))) break;
        }
        // the step that ends at a save records the nodal forces the DYNAMIC file holds
        mel_record_forces(h, euler ? (save_due ? 1 : 0) : 1);
        io.nsteps = 1;
        io.run_proximity = 1;
        if ((rc = mel_step(h, &io))) break;
        mel_record_forces(h, 0);
        number_iteration += k;
        time = io.time;
        dt = io.dt;
        if (monitoring) {
            int n = 0;
            if ((rc = mel_monitor_rows(h, rows.data(), chunk, &n))) break;
            held.insert(held.end(), rows.begin(), rows.begin() + (size_t)n * (row_len + 1));
        }
        if (time > next_print - 1.e-6 * dt) {                    // Code/main.cpp:201-206
            number_print = number_print + 1;
            next_print = next_print + run.print_period;
        }
        if (time > next_save - 1.e-6 * dt) {                     // Code/main.cpp:211-222
            number_save = number_save + 1;
            next_save = next_save + run.save_period;
            mel_save_info si = { run.simulation_name, number_save, number_iteration, number_print, next_save, next_print };
            if ((rc = mel_write_dynamic(h, dir.c_str(), &si))) break;
            if (monitoring) {
                // Write_monitoring (Code/IO.h:2644-2668)
                std::ofstream M(dir + "/MONITORING.asc", std::ios::app);
                M << std::setprecision(10);
                for (size_t r = 0; r < held.size(); r += row_len + 1) {
                    const int L = (int)held[r];
                    for (int j = 1; j <= L; j++) M << held[r + j] << ' ';
                    M << std::endl;
                }
                held.clear();
                if (!M) { std::fprintf(stderr, "cannot write %s/MONITORING.asc\n", dir.c_str()); mel_destroy(h); return 1; }
            }
        }
    }
    if (rc) {
        int code = fail("mel_step / output", rc);
        mel_destroy(h);
        return code;
    }
    mel_destroy(h);
    return 0;
}
