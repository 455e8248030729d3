// melody_gpu: host main of the B200 solver, the same shape as the reference's Code/main.cpp:25-239.
//
//   melody_gpu <restart_index> [case_dir] [steps_per_call]
//
// Reads STATIC_CONTROL.asc / STATIC_DATA.asc / DYNAMIC_<restart>.asc from case_dir (default: the
// current directory, as the reference), runs the set-up (Code/main.cpp:104-127) and then the time
// loop until Tend.  The solver and the proximity cadence run on the GPU through include/melgpu.h; the
// host reads the monitored quantities back every `steps_per_call` iterations and appends them to
// MONITORING_GPU.asc (time, dt, kinetic energy, mean displacement, rigid-body contact forces and
// driven-DOF reactions, active contacts).  Exit status is non-zero on any solver error, including
// non-finite state (the reference's NaN check, Code/main.cpp:227-237).
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <string>
#include "melgpu.h"

static int fail(const char* what, mel_status rc)
{
    std::fprintf(stderr, "%s failed (%d): %s\n", what, (int)rc, mel_last_error_string());
    return 1;
}

int main(int argc, char** argv)
{
    if (argc < 2) {
        std::fprintf(stderr, "usage: %s restart_index [case_dir] [steps_per_call]\n", argv[0]);
        return 2;
    }
    int restart = std::atoi(argv[1]);
    std::string dir = argc > 2 ? argv[2] : ".";
    int chunk = argc > 3 ? std::atoi(argv[3]) : 100;
    if (chunk < 1) chunk = 1;

    mel_model_desc* desc = nullptr;
    void* owner = nullptr;
    mel_status rc = mel_load_desc(dir.c_str(), restart, &desc, &owner);
    if (rc) return fail("mel_load_desc", rc);
    const double tend = desc->tend;
    mel_free_desc(owner);

    mel_options opt = { MEL_PREC_FP64, 0, 0, 0 };
    mel_handle* h = nullptr;
    rc = mel_create_from_files(dir.c_str(), restart, &opt, &h);
    if (rc) return fail("mel_create_from_files", rc);

    std::string mon_path = dir + "/MONITORING_GPU.asc";
    FILE* mon = std::fopen(mon_path.c_str(), "a");
    if (!mon) { std::fprintf(stderr, "cannot write %s\n", mon_path.c_str()); mel_destroy(h); return 1; }

    double time = 0., dt = 0.;
    mel_get_time(h, &time, &dt);
    long iteration = 0;
    while (time < tend) {
        mel_step_io io = {};
        io.nsteps = chunk;
        io.run_proximity = 1;
        rc = mel_step(h, &io);
        if (rc) { std::fclose(mon); mel_destroy(h); return fail("mel_step", rc); }
        iteration += chunk;
        time = io.time;
        mel_monitor m;
        rc = mel_monitor_compute(h, &m);
        if (rc) { std::fclose(mon); mel_destroy(h); return fail("mel_monitor_compute", rc); }
        std::fprintf(mon, "%ld %.17g %.17g %.17g %.17g %.17g", iteration, m.time, io.dt, m.kinetic_energy,
                     m.mean_displacement[0], m.mean_displacement[1]);
        for (int k = 0; k < 8; k++) std::fprintf(mon, " %.17g", m.rigid_force[k]);
        for (int k = 0; k < 8; k++) std::fprintf(mon, " %.17g", m.rigid_dirichlet[k]);
        std::fprintf(mon, " %d %d\n", m.active_contacts, m.n_contacts);
        if (!std::isfinite(m.kinetic_energy)) {
            std::fclose(mon);
            mel_destroy(h);
            std::fprintf(stderr, "non-finite state at iteration %ld\n", iteration);
            return (int)MEL_ERR_NAN;
        }
    }
    std::fclose(mon);
    mel_destroy(h);
    return 0;
}
