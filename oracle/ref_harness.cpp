// Test infrastructure: a driver around the reference solver, compiled from the reference's own
// headers where they lie (the include path is given by oracle/Makefile; nothing is copied).
// It repeats the set-up and loop of Code/main.cpp:88-238 without file output, and dumps the
// full state in binary at a requested cadence so the restated oracle (oracle/mel_oracle.c) and
// the GPU solver can be compared with the reference at full FP64 precision (the reference's own
// DYNAMIC files keep only 10 significant digits, Code/IO.h:2396).
//
// usage: ref_harness <case_dir> <nsteps> <dump_file> <dump_every> [threads]
//   dump records: after set-up (step 0), after each multiple of dump_every, and around every
//   proximity update (tag 0 = before Update_proximity, tag 1 = after).
// environment: REF_RESTART=k starts from DYNAMIC_k (argv[1] of Code/main.cpp); REF_OUTPUTS=1 also
//   runs the loop's output steps (Code/main.cpp:170-222): Monitoring every iteration unless
//   NO_MONITORING, the print counter, and at each save Write_dynamic and Write_monitoring, which
//   write DYNAMIC_nnnnn.asc and MONITORING.asc into case_dir as the reference does.
#include <iostream>
#include <fstream>
#include <iomanip>
#include <vector>
#include <string>
#include <sstream>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstdint>
#include <algorithm>
#include <omp.h>
#include <unistd.h>
#include <chrono>
using namespace std ;
#include "Tools.h"
#include "Material.h"
#include "Contact_Law.h"
#include "Node.h"
#include "Gauss.h"
#include "Border.h"
#include "Contact_Element.h"
#include "Body.h"
#include "Spy.h"
#include "IO.h"
#include "Solver.h"
#include "Proximity.h"
#include "Graphic.h"
#include "Monitoring.h"

static FILE* g_dump = nullptr;

static void wi(int32_t v) { fwrite(&v, 4, 1, g_dump); }
static void wd(double v) { fwrite(&v, 8, 1, g_dump); }

static void dump_state(int step, int tag, double Time, double Deltat, vector<Body>& Bodies)
{
    if (!g_dump) return;
    wi(0x4D454C44); wi(step); wi(tag); wd(Time); wd(Deltat);
    wi((int32_t)Bodies.size());
    for (auto& b : Bodies) {
        int rigid = (b.type == "rigid");
        wi(rigid); wi(b.nb_nodes);
        for (int i = 0; i < b.nb_nodes; i++) {
            Node& n = b.nodes[i];
            double v[28] = { n.x_current, n.y_current, n.x_displacement, n.y_displacement,
                             n.x_velocity, n.y_velocity, n.x_acceleration, n.y_acceleration,
                             n.x_displacement_parameter, n.y_displacement_parameter,
                             n.x_velocity_parameter, n.y_velocity_parameter,
                             n.x_acceleration_parameter, n.y_acceleration_parameter,
                             n.x_internal_force, n.y_internal_force, n.x_contact_force, n.y_contact_force,
                             n.x_body_force, n.y_body_force, n.x_dirichlet_force, n.y_dirichlet_force,
                             n.x_neumann_force, n.y_neumann_force, n.x_damping_force, n.y_damping_force,
                             n.x_force, n.y_force };
            fwrite(v, 8, 28, g_dump);
        }
        double r[30] = { b.x_current, b.y_current, b.r_current, b.x_displacement, b.y_displacement, b.r_displacement,
                         b.x_velocity, b.y_velocity, b.r_velocity, b.x_acceleration, b.y_acceleration, b.r_acceleration,
                         b.x_contact_force, b.y_contact_force, b.r_contact_force, b.x_body_force, b.y_body_force, b.r_body_force,
                         b.x_dirichlet_force, b.y_dirichlet_force, b.r_dirichlet_force,
                         b.x_neumann_force, b.y_neumann_force, b.r_neumann_force,
                         b.x_force, b.y_force, b.r_force, b.mass, b.inertia, 0.0 };
        fwrite(r, 8, 30, g_dump);
        double w[7] = { b.internal_work, b.contact_work, b.body_work, b.dirichlet_work, b.neumann_work,
                        b.damping_work, b.alid_work };
        fwrite(w, 8, 7, g_dump);
        wi(b.nb_borders);
        for (int j = 0; j < b.nb_borders; j++) {
            Border& br = b.borders[j];
            wi(br.number_border_nodes);
            for (int k = 0; k < br.number_border_nodes; k++) wd(br.length[k]);
            for (int k = 0; k < br.number_border_nodes; k++) wd(k < (int)br.x_contact_pressure.size() ? br.x_contact_pressure[k] : 0.0);
            for (int k = 0; k < br.number_border_nodes; k++) wd(k < (int)br.y_contact_pressure.size() ? br.y_contact_pressure[k] : 0.0);
        }
        wi(b.nb_neighbours);
        for (int k = 0; k < b.nb_neighbours; k++) { wi(b.neighbours[k][0]); wi(b.neighbours[k][1]); wi(b.neighbours[k][2]); }
        wi(b.nb_contact_elements);
        for (int k = 0; k < b.nb_contact_elements; k++) {
            Contact_element& c = b.contact_elements[k];
            int32_t iv[16] = { c.borderS, c.border_nodeS, c.nodeS, c.bodyM, c.borderM, c.shiftM, c.segmentM,
                               c.nodeM0, c.nodeM1, c.nodeM2, c.nodeM3, c.shiftM0, c.shiftM1, c.shiftM2, c.shiftM3,
                               c.nb_internal };
            fwrite(iv, 4, 16, g_dump);
            double dv[20] = { c.shapeM0, c.shapeM1, c.shapeM2, c.shapeM3, c.gapn, c.vgapn, c.gapt, c.vgapt, c.xsi,
                              c.xnorm, c.ynorm, c.xtan, c.ytan, c.effective_mass, c.length, c.fx, c.fy,
                              c.internal.size() > 0 ? c.internal[0] : 0.0,
                              c.internal.size() > 1 ? c.internal[1] : 0.0,
                              c.internal.size() > 2 ? c.internal[2] : 0.0 };
            fwrite(dv, 8, 20, g_dump);
        }
    }
    fflush(g_dump);
}

int main(int argc, char** argv)
{
    if (argc < 5) {
        fprintf(stderr, "usage: %s case_dir nsteps dump_file dump_every [threads]\n", argv[0]);
        return 2;
    }
    std::string dump_path = argv[3];
    if (dump_path[0] != '/' && dump_path != "-") {
        char cwd[4096];
        if (getcwd(cwd, sizeof cwd)) dump_path = std::string(cwd) + "/" + dump_path;
    }
    if (chdir(argv[1]) != 0) { perror("chdir"); return 2; }
    int nsteps = atoi(argv[2]);
    int every = atoi(argv[4]);
    if (argc > 5) omp_set_num_threads(atoi(argv[5]));
    if (dump_path != "-") {
        g_dump = fopen(dump_path.c_str(), "wb");
        if (!g_dump) { perror("dump"); return 2; }
    }
    std::streambuf* oldbuf = std::cout.rdbuf();
    std::ofstream devnull("/dev/null");
    std::cout.rdbuf(devnull.rdbuf());

    string Simulation_name ;
    int Nb_materials ;
    vector<Material> Materials ;
    int Nb_contact_laws ;
    vector<Contact_law> Contact_laws ;
    string Solver ;
    double Tini, Deltat, Tend, Time ;
    double Target_error = 0, Inv_Target_error = 0, Control_parameter = 0, Accepted_ratio = 0 ;
    double Max_mass_scaling = 0, Control_parameter_mass_scaling = 0, Error_factor_mass_scaling = 0, Decrease_factor_mass_scaling = 0 ;
    double Save_period, Print_period, Contact_update_period ;
    double Next_save, Next_print, Next_contact_update ;
    int Number_save(0), Number_print, Number_iteration ;
    double Xmin_period, Xmax_period, Penalty = 0 ;
    double Xgravity, Ygravity ;
    int Activate_plot = 0 ;
    double Xmin_plot = 0, Xmax_plot = 0, Ymin_plot = 0, Ymax_plot = 0 ;
    int Nb_bodies ;
    vector<Body> Bodies ;
    int Nb_monitored = 0 ;
    vector<vector<double>> Monitored ;
    int Nb_deactivated = 0 ;
    vector<vector<double>> Deactivated ;
    int Nb_spies = 0 ;
    vector<Spy> Spies ;
    int neval = 0 ;
    double max_error = 0, mean_error = 0 ;
    double total_mass = 0, max_mass = 0 ;
    int Nb_regions = 0 ;
    vector<vector<int>> Regions ;
    vector<int> flags(11) ;
    vector<int> To_Plot(41) ;
    vector<vector<int>> Contacts_Table ;

    Load_static( Simulation_name, Nb_materials, Materials, Nb_contact_laws, Contact_laws, Contacts_Table,
                 Solver, Tini, Deltat, Tend, Target_error, Inv_Target_error, Control_parameter, Accepted_ratio,
                 Max_mass_scaling, Control_parameter_mass_scaling, Error_factor_mass_scaling, Decrease_factor_mass_scaling,
                 Save_period, Print_period, Contact_update_period, Xmin_period, Xmax_period, Penalty, Xgravity, Ygravity,
                 Activate_plot, Xmin_plot, Xmax_plot, Ymin_plot, Ymax_plot,
                 Nb_monitored, Monitored, Nb_deactivated, Deactivated, Nb_spies, Spies,
                 Nb_regions, Regions, Nb_bodies, Bodies, To_Plot ) ;
    Number_save = getenv("REF_RESTART") ? atoi(getenv("REF_RESTART")) : 0 ;
    const bool outputs = getenv("REF_OUTPUTS") && atoi(getenv("REF_OUTPUTS")) == 1 ;
    vector<vector<double>> monitoring ;
    Load_dynamic( Number_save, Number_print, Time, Number_iteration, Deltat, Solver,
                  Next_save, Next_print, Next_contact_update, Xmin_period, Xmax_period, Bodies, flags ) ;
    // set-up of Code/main.cpp:104-127
    for (int i=0 ; i<Nb_bodies ; i++) Bodies[i].Update_borders(Xmin_period, Xmax_period) ;
    for (int i=0 ; i<Nb_bodies ; i++) Bodies[i].Update_bc(Time) ;
    Update_proximity(Nb_bodies, Bodies, Xmin_period, Xmax_period, flags) ;
    if (flags[3]==1) Initialize_CZM( Nb_bodies, Bodies, Nb_contact_laws, Contact_laws, flags, Xmin_period, Xmax_period ) ;
    #pragma omp parallel
    {
        #pragma omp for schedule(dynamic)
        for (int i=0 ; i<Nb_bodies ; i++) Bodies[i].Update_material( Nb_materials, Materials, flags ) ;
    }
    Update_proximity(Nb_bodies, Bodies, Xmin_period, Xmax_period, flags) ;
    if (flags[3]==1) Initialize_CZM( Nb_bodies, Bodies, Nb_contact_laws, Contact_laws, flags, Xmin_period, Xmax_period ) ;
    dump_state(0, 1, Time, Deltat, Bodies);

    auto t0 = std::chrono::steady_clock::now();
    double t_prox = 0.0;
    for (int it = 1; it <= nsteps; it++) {
        Number_iteration++ ;
        if (Solver == "Euler")
            Euler_step(Nb_bodies, Bodies, Nb_regions, Regions, Nb_materials, Materials, Nb_contact_laws, Contact_laws,
                       Contacts_Table, Tend, Xmin_period, Xmax_period, Penalty, Xgravity, Ygravity,
                       Time, Deltat, Number_iteration, flags) ;
        else
            Solver_step(Nb_bodies, Bodies, Nb_regions, Regions, Nb_materials, Materials, Nb_contact_laws, Contact_laws,
                        Contacts_Table, Tend, Xmin_period, Xmax_period, Penalty, Xgravity, Ygravity,
                        Time, Deltat, Number_iteration, Next_contact_update, Contact_update_period,
                        Target_error, Inv_Target_error, Control_parameter, Accepted_ratio,
                        Max_mass_scaling, Control_parameter_mass_scaling, Error_factor_mass_scaling, Decrease_factor_mass_scaling,
                        neval, max_error, mean_error, flags, total_mass, max_mass, Solver) ;
        if (outputs && flags[8]==0)
            Monitoring(Nb_bodies, Bodies, Time, Deltat, Number_iteration, neval, max_error, mean_error, flags,
                       monitoring, Nb_monitored, Monitored) ;
        bool prox = Time > Next_contact_update-1.e-6*Deltat ;
        if (prox || (every > 0 && it % every == 0)) dump_state(it, 0, Time, Deltat, Bodies);
        if (prox) {
            auto p0 = std::chrono::steady_clock::now();
            Next_contact_update = Next_contact_update + Contact_update_period ;
            Update_proximity(Nb_bodies, Bodies, Xmin_period, Xmax_period, flags) ;
            Update_status(Nb_bodies, Bodies, Nb_deactivated, Deactivated) ;
            t_prox += std::chrono::duration<double>(std::chrono::steady_clock::now() - p0).count();
            dump_state(it, 1, Time, Deltat, Bodies);
        }
        if (outputs) {
            if ( Time > Next_print-1.e-6*Deltat ) {
                Number_print = Number_print + 1 ;
                Next_print = Next_print + Print_period ;
            }
            if ( Time > Next_save-1.e-6*Deltat ) {
                Number_save = Number_save + 1 ;
                Next_save = Next_save + Save_period ;
                Write_dynamic( Simulation_name, Number_save, Number_print, Time, Number_iteration, Deltat, Solver,
                               Next_save, Next_print, Next_contact_update, Nb_bodies, Bodies, flags ) ;
                if (flags[8]==0) Write_monitoring( monitoring, flags ) ;
            }
        }
    }
    double wall = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    std::cout.rdbuf(oldbuf);
    long nodes = 0;
    for (auto& b : Bodies) if (b.type == "deformable") nodes += b.nb_nodes;
    printf("{\"steps\": %d, \"wall_s\": %.6f, \"proximity_s\": %.6f, \"deformable_nodes\": %ld, \"threads\": %d, \"time\": %.17g}\n",
           nsteps, wall, t_prox, nodes, omp_get_max_threads(), Time);
    if (g_dump) fclose(g_dump);
    return 0;
}
