/*
 * melgpu.h -- C ABI of the B200 solver for the MELODY 2D explicit-dynamics step.
 *
 * The reference has no plugin or FFI: its step is the C++ call
 *   Euler_step(...)            Code/Solver.h:10-88   (dispatched at Code/main.cpp:148-155)
 *   Solver_step(...)           Code/Solver.h:98-486  (dispatched at Code/main.cpp:156-167)
 *   Update_proximity(...)      Code/Proximity.h:48-473 (called at Code/main.cpp:191-196)
 * operating in place on `vector<Body>` filled by Load_static (Code/IO.h:598) and
 * Load_dynamic (Code/IO.h:1871).  This header is the seam that replaces those calls:
 * a host main of the same shape as Code/main.cpp loads the same input files, hands the
 * flattened model to mel_create / mel_create_from_files, advances it with mel_step and
 * reads state back with mel_download at monitoring / save cadence.
 *
 * Conventions: plain C, host pointers and counts only; the library owns all device memory;
 * every call returns a mel_status; one host thread per handle; one CUDA stream per handle.
 * Node, border and Gauss-point indices inside a body are body-local, exactly as in the
 * reference input files.
 */
#ifndef MELGPU_H
#define MELGPU_H

#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define MELGPU_ABI_VERSION 2

/* ---- status codes ---------------------------------------------------------------- */
typedef enum {
    MEL_OK = 0,
    MEL_ERR_INVALID = 1,      /* bad argument or malformed model description          */
    MEL_ERR_UNSUPPORTED = 2,  /* valid reference input this build does not run yet    */
    MEL_ERR_CUDA = 3,         /* CUDA runtime error (message in mel_last_error_string) */
    MEL_ERR_OOM = 4,          /* device allocation failed                              */
    MEL_ERR_NAN = 5,          /* non-finite state detected (Code/main.cpp:227-237)     */
    MEL_ERR_BOUNDS = 6,       /* device-side index check failed                        */
    MEL_ERR_TIMEOUT = 7,      /* a bounded device wait gave up                         */
    MEL_ERR_IO = 8,           /* input file missing or unreadable                      */
    MEL_ERR_NO_DEVICE = 9     /* no CUDA device                                        */
} mel_status;

/* ---- enumerations mirroring the reference's string tags ---------------------------- */
enum { MEL_BODY_DEFORMABLE = 0, MEL_BODY_RIGID = 1 };                 /* Body::type        */
enum { MEL_STATUS_ACTIVE = 0, MEL_STATUS_INACTIVE = 1, MEL_STATUS_NOGRAVITY = 2 }; /* Body::status */
enum { MEL_PER_CLOSED = 0, MEL_PER_SIMPLE = 1, MEL_PER_PERIODIC = 2 };  /* Border/Body periodicity */
enum { MEL_INTERP_LINEAR = 0, MEL_INTERP_SPLINE = 1 };                 /* Border::interpolant */
enum { MEL_BC_NONE = 0, MEL_BC_SOFT = 1, MEL_BC_DRIVEN = 2, MEL_BC_ORIENTED = 3, MEL_BC_FOLLOWING = 4 };
enum { MEL_MAT_ELASTIC_LINEAR = 0, MEL_MAT_NEOHOOKEAN = 1 };
enum { MEL_LAW_FRICTIONLESS = 0, MEL_LAW_COHESION = 1, MEL_LAW_MOHR_COULOMB = 2,
       MEL_LAW_DAMPED_MOHR_COULOMB = 3, MEL_LAW_TWO_SLOPES_MOHR_COULOMB = 4,
       MEL_LAW_BONDED_MOHR_COULOMB = 5, MEL_LAW_CZM_LINEAR = 6, MEL_LAW_CZM_FATIGUE = 7 };
enum { MEL_LENGTH_FIXED = 0, MEL_LENGTH_EVOLUTIVE = 1 };
enum { MEL_SOLVER_EULER = 0, MEL_SOLVER_ADAPTIVE_EULER = 1, MEL_SOLVER_MASS_SCALING = 2,
       MEL_SOLVER_ADAPTIVE_MASS_SCALING = 3, MEL_SOLVER_EULER_2 = 4 };
/* Arithmetic of the Gauss-point pass: all-FP64 drop-in, or FP32 shape-function
 * derivatives / strain / stress with FP64 kinematics, gaps and nodal sums. */
enum { MEL_PREC_FP64 = 0, MEL_PREC_MIXED = 1 };

#define MEL_MAT_NPARAM   6   /* rho, alpha, beta, mu, lambda|kappa, heat_capacity  (Code/IO.h:672-685) */
#define MEL_LAW_NPARAM  11   /* largest law: BondedMohrCoulomb                     (Code/IO.h:775-783) */
#define MEL_RIGID_NF    20   /* see MEL_RG_* below                                                    */
#define MEL_NFLAGS      11   /* DYNAMIC flags[0..10]                               (Code/IO.h:1912-1933) */
#define MEL_NINTERNAL    3   /* Contact_element::internal values kept on device                         */
#define MEL_DEACT_NF     8   /* doubles per DEACTIVATION entry in mel_model_desc::deactivated          */

/* Layout of one rigid-body record in mel_model_desc::rigid (Body.h:46-95 rigid attributes). */
enum { MEL_RG_X0 = 0, MEL_RG_Y0, MEL_RG_R0, MEL_RG_MASS, MEL_RG_INERTIA, MEL_RG_INV_MASS, MEL_RG_INV_INERTIA,
       MEL_RG_XC, MEL_RG_YC, MEL_RG_RC, MEL_RG_XD, MEL_RG_YD, MEL_RG_RD, MEL_RG_XV, MEL_RG_YV, MEL_RG_RV,
       MEL_RG_XA, MEL_RG_YA, MEL_RG_RA, MEL_RG_PAD };

/* Flattened model: the content of STATIC_CONTROL.asc + STATIC_DATA.asc + DYNAMIC_nnnnn.asc
 * after Load_static / Load_dynamic, as structure-of-arrays.  All arrays are host memory
 * owned by the caller and only read during mel_create. */
typedef struct mel_model_desc {
    int    abi_version;                 /* = MELGPU_ABI_VERSION */
    /* scene (Code/IO.h:821-915, 1944-1953) */
    double period[2];                   /* Xmin_period, Xmax_period */
    double gravity[2];                  /* Xgravity, Ygravity */
    double time, dt, tend;
    double contact_update_period, next_contact_update;
    int    solver;                      /* MEL_SOLVER_* */
    double solver_params[8];            /* Target_error, Control_parameter, Accepted_ratio, Max_mass_scaling,
                                           Control_parameter_mass_scaling, Error_factor_mass_scaling,
                                           Decrease_factor_mass_scaling, Inv_Target_error */
    int    flags[MEL_NFLAGS];
    /* materials and contact laws (Code/IO.h:660-812) */
    int           n_materials;
    const int*    material_type;        /* [n_materials] MEL_MAT_* */
    const double* material_params;      /* [n_materials*MEL_MAT_NPARAM] */
    int           n_laws;
    const int*    law_type;             /* [n_laws] MEL_LAW_* */
    const int*    law_length;           /* [n_laws] MEL_LENGTH_* */
    const double* law_params;           /* [n_laws*MEL_LAW_NPARAM] */
    const int*    contacts_table;       /* [n_materials*n_materials], -1 = no law */
    /* bodies (Code/IO.h:1013-1070, 1494-1520) */
    int           n_bodies;
    const int*    body_type;            /* MEL_BODY_* */
    const int*    body_material;
    const int*    body_periodic;        /* 1 when the body's type string is "Periodic" */
    const int*    body_status;          /* MEL_STATUS_* */
    const double* body_dist;            /* [n_bodies*3] nodal, detection, contact distance */
    const int*    body_node_ptr;        /* [n_bodies+1] into node arrays */
    const int*    body_border_ptr;      /* [n_bodies+1] into border arrays */
    const int*    body_gp_ptr;          /* [n_bodies+1] into Gauss-point arrays */
    const int*    body_cell_ptr;        /* [n_bodies+1] into cells */
    const double* rigid;                /* [n_bodies*MEL_RIGID_NF] (ignored for deformable bodies) */
    /* nodes of all bodies, body-contiguous (Node.h, Code/IO.h:1522-1630, 1796-1830) */
    int           n_nodes;
    const double* node_x0;              /* [2*n_nodes] x_initial, y_initial */
    const double* node_mass;            /* [2*n_nodes] x_mass, y_mass */
    const double* node_inv_mass;        /* [2*n_nodes] */
    const double* node_domain;          /* [n_nodes] domain_size */
    const int*    node_sup_ptr;         /* [n_nodes+1] DOF_TO_DISP supports (empty for rigid nodes) */
    const int*    node_sup_idx;         /* body-local */
    const double* node_sup_N;           /* shape function values */
    const double* node_state;           /* [n_nodes*12]: u x,y  v x,y  a x,y  up x,y  vp x,y  ap x,y */
    /* borders (Border.h; Code/IO.h:1072-1290, 1632-1660) */
    int           n_borders;
    const int*    border_body;
    const int*    border_periodicity;   /* MEL_PER_* */
    const int*    border_interpolant;   /* MEL_INTERP_* */
    const int*    border_before;        /* body-local border index */
    const int*    border_after;
    const int*    border_node_ptr;      /* [n_borders+1] */
    const int*    border_nodes;         /* body-local node index per border node */
    const int*    border_bc_type;       /* [2*n_borders] x then y, MEL_BC_* */
    const double* border_bc_param;      /* [4*n_borders] soft penalty,damping for x then y */
    const int*    border_hist_ptr;      /* [2*n_borders+1] history of (border,dir) k is [ptr[k],ptr[k+1]) */
    const double* hist_time;
    const double* hist_value;
    /* Gauss points (Code/IO.h:1662-1760) */
    int           n_gauss;
    const int*    gp_sup_ptr;           /* [n_gauss+1] */
    const int*    gp_sup_idx;           /* body-local */
    const double* gp_N;
    const double* gp_dNdx;
    const double* gp_dNdy;
    const double* gp_weight;            /* [n_gauss] */
    const double* gp_jacobian;          /* [n_gauss] */
    /* background triangulation (rigid mass and inertia, Body.h:2871-2897) */
    int           n_cells;
    const int*    cells;                /* [3*n_cells] body-local */
    /* damping matrix triplets (Code/IO.h:1832-1855): dof0, dof1 body-local dofs */
    int           n_matrix;
    const int*    body_matrix_ptr;      /* [n_bodies+1] or NULL when n_matrix == 0 */
    const int*    matrix_dofs;          /* [2*n_matrix] */
    const double* matrix_stiffness;     /* as in the file: with flags[5] / flags[6] (UPDATE_STIFFNESS_MATRIX, */
    const double* matrix_damping;       /* UPDATE_DAMPING_MATRIX) mel_create rebuilds its own copies from the
                                           material (Body::Update_material, Code/Body.h:2784-2875) */
    /* DEACTIVATION entries of STATIC_CONTROL (Code/IO.h:947-968): the vector Read_spy_line builds,
     * then the comparison (0 below, 1 equal, 2 above) and the threshold, zero-padded to
     * MEL_DEACT_NF doubles; Update_status (Code/Proximity.h:550-1007) applies them after every
     * proximity update */
    int           n_deactivated;
    const double* deactivated;          /* [n_deactivated*MEL_DEACT_NF] or NULL */
    /* ALID absorbing layers (the ALID block of STATIC_CONTROL, Code/IO.h:1395-1480): per body and
     * direction the history of the layer's reference velocity (a body has a layer when either
     * history is non-empty), and per node alid_alpha and alid_beta as Load_static computes them
     * from the node's initial position (Code/IO.h:1548-1600).  Body::Update_alid_forces
     * (Code/Body.h:1163-1296) also uses the body's matrix_stiffness entries.  All NULL when no
     * body has a layer. */
    const int*    body_alid_ptr;        /* [2*n_bodies+1]: history of (body, dir) k is [ptr[k], ptr[k+1]) */
    const double* alid_time;
    const double* alid_value;
    const double* node_alid;            /* [2*n_nodes] alid_alpha, alid_beta */
} mel_model_desc;

/* One contact element (Contact_Element.h:5-55) in the reference's own field order. */
typedef struct mel_contact {
    int32_t bodyS, borderS, border_nodeS, nodeS;
    int32_t bodyM, borderM, shiftM, segmentM;
    int32_t nodeM[4], shiftMk[4];
    double  shapeM[4];
    double  gapn, vgapn, gapt, vgapt, xsi, xnorm, ynorm, xtan, ytan;
    double  effective_mass, length, fx, fy;
    int32_t nb_internal, pad_;
    double  internal[MEL_NINTERNAL];
} mel_contact;

/* Step parameters and outputs of mel_step. */
typedef struct mel_step_io {
    int    nsteps;          /* accepted steps to take */
    int    run_proximity;   /* 1: run Update_proximity when Time >= Next_contact_update (Code/main.cpp:191) */
    double time;            /* out: Time after the call */
    double dt;              /* out: Deltat after the call */
    double next_contact_update; /* out */
    int    n_contacts;      /* out: contact elements after the call */
    int    n_proximity;     /* out: proximity updates performed */
} mel_step_io;

/* Parity quantities reduced on the device (Code/Monitoring.h). */
typedef struct mel_monitor {
    double time;
    double kinetic_energy;          /* Σ ½ m v² over nodal velocities  (Monitoring.h:528-531) */
    double mean_displacement[2];    /* mass-weighted over deformable nodes (Monitoring.h:88-101) */
    double rigid_force[2*4];        /* first four rigid bodies: Σ contact force x,y  */
    double rigid_dirichlet[2*4];    /* first four rigid bodies: driven-DOF reaction x,y (Body.h:2093,2105) */
    int    active_contacts;         /* contact elements with nonzero force */
    int    n_contacts;
} mel_monitor;

typedef struct mel_options {
    int precision;          /* MEL_PREC_* */
    int device;             /* CUDA device ordinal */
    int use_graph;          /* reserved, must be 0 */
    int max_contacts;       /* reserved, must be 0 (contact storage grows as needed) */
} mel_options;

typedef struct mel_handle mel_handle;

/* ---- lifecycle -------------------------------------------------------------------- */
/* Replaces Load_static + Load_dynamic + the initialisation block of Code/main.cpp:104-127
 * (Update_borders, Update_bc, Update_proximity x2, Update_material). */
mel_status mel_create(const mel_model_desc* desc, const mel_options* opt, mel_handle** out);
/* Same, reading STATIC_CONTROL.asc / STATIC_DATA.asc / DYNAMIC_nnnnn.asc from `dir`
 * (Code/IO.h:598, Code/IO.h:1871; `restart_index` is argv[1] of Code/main.cpp:94). */
mel_status mel_create_from_files(const char* dir, int restart_index, const mel_options* opt, mel_handle** out);
mel_status mel_destroy(mel_handle* h);

/* ---- stepping --------------------------------------------------------------------- */
/* io->nsteps iterations of the loop body of Code/main.cpp:141-238 restricted to the solver and the
 * proximity update (Code/main.cpp:191-196): Euler_step (Code/Solver.h:10-88) for MEL_SOLVER_EULER,
 * Solver_step (Code/Solver.h:98-486: two half-steps, error estimate, mass scaling, accept / reject
 * with Deltat control) for the other schemes; io->nsteps counts accepted steps. */
mel_status mel_step(mel_handle* h, mel_step_io* io);
/* Update_proximity (Code/Proximity.h:48-473) on the current positions. */
mel_status mel_update_proximity(mel_handle* h);
/* Replace the contact list (restart or host-side proximity; mirrors Load_dynamic CONTACTS). */
mel_status mel_set_contacts(mel_handle* h, const mel_contact* contacts, int n);

/* ---- state transfer --------------------------------------------------------------- */
/* node_state layout as in mel_model_desc::node_state (12 doubles per node). */
mel_status mel_get_node_state(mel_handle* h, double* node_state);
mel_status mel_set_node_state(mel_handle* h, const double* node_state);
/* Page-lock (pin) a caller-owned host buffer, so that the state transfers above and below move at
 * the host link's full speed instead of through a pageable bounce; mel_unpin_host releases it.
 * No counterpart in the reference, whose state lives in host memory only. */
mel_status mel_pin_host(void* ptr, size_t bytes);
mel_status mel_unpin_host(void* ptr);
/* current positions, 2 doubles per node */
mel_status mel_get_positions(mel_handle* h, double* xy);
/* nodal force components of the last step, [n_nodes*2] each; any pointer may be NULL.
 * internal = Σ regions internal force (Node.h:216-222), contact, neumann, dirichlet, total. */
mel_status mel_get_forces(mel_handle* h, double* internal, double* contact, double* neumann,
                          double* dirichlet, double* total);
mel_status mel_get_rigid(mel_handle* h, double* rigid /* [n_bodies*MEL_RIGID_NF] */,
                         double* rigid_forces /* [n_bodies*12]: contact, body, dirichlet, neumann (x,y,r) */);
/* works per body [n_bodies*7]: internal, contact, body, dirichlet, neumann, damping, alid (Body.h:111-117) */
mel_status mel_get_works(mel_handle* h, double* works);
mel_status mel_get_contact_count(mel_handle* h, int* n);
/* Solver_step statistics of the last accepted step (Code/Solver.h:98-486): attempts (neval),
 * max_error, mean_error, total_mass, max_mass; zeros under the Euler scheme. */
mel_status mel_get_solver_stats(mel_handle* h, double* out5);
/* Border contact pressures of the last step, x and y, one per border entry in the order of the
 * border node lists (Update_contact_pressures, Code/Proximity.h:1014-1069, which the reference runs
 * at the end of every accepted step; Border::x_contact_pressure, y_contact_pressure).  They are
 * computed when first asked for after a step, or before the proximity update that would replace
 * the contact list they come from; a batch member keeps them across such updates only with
 * mel_record_forces on. */
mel_status mel_get_contact_pressures(mel_handle* h, double* px, double* py);
mel_status mel_get_contacts(mel_handle* h, mel_contact* out, int capacity, int* n);
/* Body statuses (MEL_STATUS_*, n_bodies values): Update_status (Code/Proximity.h:550-1007) turns
 * bodies inactive after a proximity update when a DEACTIVATION entry's condition holds. */
mel_status mel_get_body_status(mel_handle* h, int* status);
mel_status mel_get_time(mel_handle* h, double* time, double* dt);

/* Asynchronous checkpoint (replaces the blocking downloads that precede Write_dynamic,
 * Code/IO.h:2351, when the host keeps stepping meanwhile).  mel_checkpoint_start snapshots the
 * node state, rigid records, works, contact list and time on the handle's stream (it sees every
 * step called before it and none after) and copies it to library-owned pinned memory on a side
 * stream; it returns without waiting, and further mel_step calls overlap the copy.
 * mel_checkpoint_read waits for the copy and fills the caller's buffers (any may be NULL):
 * node_state as mel_get_node_state, rigid as mel_get_rigid, works as mel_get_works, contacts (up
 * to contacts_capacity records; too small a buffer is an error that leaves the snapshot pending),
 * *ncont, and time3 = {time, dt, next_contact_update}.  A second start before a read replaces
 * the unread snapshot.  For a batch member the snapshot is completed before start returns. */
mel_status mel_checkpoint_start(mel_handle* h);
mel_status mel_checkpoint_read(mel_handle* h, double* node_state, double* rigid, double* works,
                               mel_contact* contacts, int contacts_capacity, int* ncont, double* time3);
mel_status mel_monitor_compute(mel_handle* h, mel_monitor* out);

/* Border-condition pressures of the last step, x and y, one per border entry in the order of the
 * border node lists (Border::x_bc_pressure, y_bc_pressure, set by Update_bc_forces,
 * Code/Body.h:669-901; zero on borders whose conditions are both none). */
mel_status mel_get_bc_pressures(mel_handle* h, double* px, double* py);

/* ---- monitoring and reference-format output ------------------------------------------ */
#define MEL_MON_NF 7   /* doubles per monitored entry: the vector Read_spy_line builds (Code/IO.h:11-590), zero-padded */
/* Monitoring (Code/Monitoring.h:8-559) on the device: after every accepted step of mel_step one row
 * is appended to a device buffer of ring_rows rows, without a host download, until
 * mel_monitor_rows drains it (the reference keeps rows in memory and flushes them at save time,
 * Code/IO.h:2644-2668).  `monitored` holds n_monitored entries of MEL_MON_NF doubles, the rows of the
 * reference's Monitored array as Read_spy_line builds them from STATIC_CONTROL's MONITORING section
 * (mel_load_run fills them); monitor_energy and monitor_boundaries are DYNAMIC flags[1] and flags[2];
 * first_iteration is Number_iteration before the next step.  A row holds Number_iteration, Time,
 * Deltat, neval, max_error, mean_error (the last three are 0 under the Euler scheme, which never
 * sets them), one value per entry that yields one, then Dwork, elastic energy and kinetic energy
 * (monitor_energy) and the four boundary sums (monitor_boundaries).  Contact entries yield a value
 * only while their slave node has a contact element, so rows can differ in length;
 * *max_row_length receives the longest.  Entry types 5 (Jacobian), 6 (Stress) and 8 (Damage) need
 * the nodal stress post-processing or Body::Update_damage, which this library does not run:
 * MEL_ERR_UNSUPPORTED.  Force entries of nodes or deformable bodies keep mel_record_forces on.
 * Entries are checked against the model (the reference indexes its arrays with them unchecked):
 * out of range is MEL_ERR_INVALID.  n_monitored = 0 with both flags 0 turns monitoring off.  A
 * batch member cannot monitor (MEL_ERR_INVALID).  mel_step refuses (MEL_ERR_INVALID, nothing done)
 * to take more steps than the buffer has free rows. */
mel_status mel_monitor_setup(mel_handle* h, const double* monitored, int n_monitored, int monitor_energy,
                             int monitor_boundaries, int ring_rows, int first_iteration, int* max_row_length);
/* The rows recorded since the last call, oldest first, and empties the buffer: row i occupies
 * rows[i*(max_row_length+1) ...], its first double the number L of values that follow.
 * rows = NULL with max_rows = 0 only sets *n_rows to the number held.  A buffer of fewer than
 * *n_rows rows is MEL_ERR_INVALID and drains nothing (*n_rows says how many are held). */
mel_status mel_monitor_rows(mel_handle* h, double* rows, int max_rows, int* n_rows);

/* What the input files say about output (Code/IO.h:598-2345), for a host loop that writes the
 * reference's files: Simulation_name, Save_period and Print_period (STATIC_CONTROL SOLVER block),
 * Number_save, Number_iteration, Number_print, Next_save, Next_print (DYNAMIC SOLVER block), the
 * MONITORING entries (Code/IO.h:933-945, the vectors Read_spy_line builds, zero-padded to
 * MEL_MON_NF) and the DYNAMIC flags. */
#define MEL_MON_MAX 256
typedef struct mel_run_control {
    char   simulation_name[256];
    double save_period, print_period, next_save, next_print;
    int    number_save, number_iteration, number_print;
    int    n_monitored;
    double monitored[MEL_MON_MAX * MEL_MON_NF];
    int    flags[MEL_NFLAGS];
} mel_run_control;
/* Fills *out from a model read by mel_load_desc (its owner). */
mel_status mel_load_run_control(const void* owner, mel_run_control* out);
/* mel_create from a model read by mel_load_desc, with the contact list of its DYNAMIC file (as
 * mel_create_from_files, without reading the files again). */
mel_status mel_create_loaded(const void* owner, const mel_options* opt, mel_handle** out);

/* Run counters of Code/main.cpp that Write_dynamic records but the solver does not keep. */
typedef struct mel_save_info {
    const char* simulation_name;
    int    number_save;       /* the file is DYNAMIC_<number_save, 5 digits>.asc */
    int    number_iteration;
    int    number_print;
    double next_save, next_print;
} mel_save_info;
/* Write_dynamic (Code/IO.h:2351-2640): writes <dir>/DYNAMIC_nnnnn.asc from the handle's state in
 * the reference's layout and number formatting (what Load_dynamic and mel_create_from_files read
 * back to restart): kinematics, forces, works, neighbours, border segments, contact elements,
 * contact and border-condition pressures, and the Time, Deltat and Next_contact_update of the
 * handle.  The FORCES blocks are the nodal forces of the last step, so mel_record_forces must have
 * been on during it (MEL_ERR_INVALID otherwise); the self-contact components are zero, as the
 * reference never fills them. */
mel_status mel_write_dynamic(mel_handle* h, const char* dir, const mel_save_info* info);

/* Rigid-body records (layout MEL_RG_*, n_bodies records); node positions follow (restart upload). */
mel_status mel_set_rigid(mel_handle* h, const double* rigid);
/* Time, Deltat and Next_contact_update of the loop (Code/IO.h:1944-1953; restart upload). */
mel_status mel_set_time(mel_handle* h, double time, double dt, double next_contact_update);
/* Keep per-node force components of each step for mel_get_forces (off by default: extra writes). */
mel_status mel_record_forces(mel_handle* h, int on);
/* Time each launch of mel_step with CUDA events on the handle's stream (mel_get_kernel_times). */
mel_status mel_set_timing(mel_handle* h, int on);
/* Device diagnostic words: [0] index checks, [1] neighbour overflow, [2] contacts whose projection
 * weights the reference would take from another contact (Code/Body.h:1347), ... */
mel_status mel_get_error_words(mel_handle* h, unsigned* words, int n);
/* Parse the input files into a mel_model_desc owned by the library (release with mel_free_desc). */
mel_status mel_load_desc(const char* dir, int restart_index, mel_model_desc** desc, void** owner);
mel_status mel_free_desc(void* owner);

/* Monitored quantities from caller-held device arrays, allocating no device memory.
 * This entry point has no counterpart in the reference (its monitoring runs on the host,
 * Code/Monitoring.h).  It serves callers that cannot allocate device memory themselves -- a
 * framework or runtime that owns all device memory through its own allocator, or a deployment with
 * a fixed device-memory budget -- and already hold the state on the device.  Inputs (device):
 * velocity, mass and displacement as x,y pairs for n_nodes nodes, and n_contacts contact elements;
 * output (device): d_out[0..3] = kinetic energy, mean displacement x and y (mass-weighted), number
 * of contact elements with a nonzero force -- the quantities mel_monitor_compute reports.
 * Its block partials live in a file-scope device array of 1024 records reused by every call (and
 * held by every GPU that loads the library until the process exits), so it accepts at most
 * 2,097,152 nodes and as many contact elements per call and rejects larger sizes with
 * MEL_ERR_INVALID.  The array keeps the last call's contents; each call writes every record it reads,
 * and calls that overlap on the GPU (on different streams) race on it.  Each call looks up the
 * array's device address in the current device's context, so the address stays right after a device
 * reset; the first call on a device loads the library's device code, so make that first call before
 * any stream capture.  A CUDA error already pending from the caller's own launches is reported as
 * MEL_ERR_CUDA and left pending, and nothing is launched.  `stream` is a cudaStream_t (NULL: the
 * legacy default stream); the call returns once the work is queued. */
mel_status mel_monitor_reduce_static(const double* d_velocity, const double* d_mass, const double* d_displacement,
                                     int n_nodes, const mel_contact* d_contacts, int n_contacts, double* d_out,
                                     void* stream);

/* ---- input generation ------------------------------------------------------------------ */
/* Shape functions and derivatives at the Gauss points of n_bodies bodies, computed on the device:
 * the moving-least-squares pass of the reference's pre-processor with the linear basis
 * (Preprocessor/MLS2DWithDerivatives.m:65-165), the cubic-spline weight W1
 * (Preprocessor/WeightW1WithDerivatives.m:17-47) and the support rule |x_p - x_i| < r_i
 * (Preprocessor/SupportDomain.m:16-18).  Host arrays: body b owns nodes [body_node_ptr[b],
 * body_node_ptr[b+1]) (x,y pairs in `nodes`, influence radii in `radii`) and Gauss points
 * [body_point_ptr[b], body_point_ptr[b+1]) (x,y pairs in `points`), at most 4096 nodes per body.
 * Output in CSR: sup_ptr[n_points+1] offsets, then per entry the body-local support node (ascending
 * within a point, as SupportDomain lists them), N, dN/dx, dN/dy -- the layout of
 * mel_model_desc::gp_sup_*, gp_N, gp_dNdx, gp_dNdy.  Call with sup_idx = NULL to get sup_ptr and
 * *n_entries only; then with buffers of `capacity` >= *n_entries entries.  A point whose supports
 * do not span the plane (singular moment matrix) is MEL_ERR_INVALID, naming it.  kernel_ms (may be
 * NULL) receives the device time of the value pass.  No counterpart in the solver (the reference
 * computes these in MATLAB before the run). */
mel_status mel_mls_shapes(int n_bodies, const int* body_node_ptr, const double* nodes, const double* radii,
                          const int* body_point_ptr, const double* points, long long* sup_ptr, int* sup_idx,
                          double* N, double* dNdx, double* dNdy, long long capacity, long long* n_entries, int device,
                          double* kernel_ms);

/* ---- batches ------------------------------------------------------------------------ */
/* No counterpart in the reference (one simulation per process there).  A batch advances several
 * independent handles (samples) with shared launches: per step one contact pass over all members'
 * contact elements, one body pass over all members' bodies and one time advance, so many small
 * samples fill the GPU together.  Each member keeps its own device arrays, time, dt and proximity
 * cadence (Code/main.cpp:191-196, run per member on the batch's stream when its time comes), and
 * computes exactly what mel_step would compute for it alone.  Members are admitted and retired
 * between steps (continuous batching); a member cannot be stepped with mel_step, and mel_destroy
 * retires it first.  All members share the batch's device and precision. */
typedef struct mel_batch mel_batch;
mel_status mel_batch_create(int device, int precision, mel_batch** out);
mel_status mel_batch_admit(mel_batch* b, mel_handle* h);
mel_status mel_batch_retire(mel_batch* b, mel_handle* h);
/* nsteps steps of every member; run_proximity as in mel_step_io.  Returns after the work is done.
 * A member whose state diverges (MEL_ERR_NAN at its proximity update) or fails a device index check
 * leaves the batch and the others carry on; mel_get_health reports it. */
mel_status mel_batch_step(mel_batch* b, int nsteps, int run_proximity);
/* *failed = 0 for a healthy handle, else the status that retired it from its batch (the message is
 * then available from mel_last_error_string). */
mel_status mel_get_health(mel_handle* h, int* failed);
/* device time of the last mel_batch_step call (CUDA events), kernels it launched, current members */
mel_status mel_batch_stats(mel_batch* b, double* ms_last_call, long long* launches, int* members);
mel_status mel_batch_destroy(mel_batch* b);

/* ---- introspection ---------------------------------------------------------------- */
const char* mel_last_error_string(void);
int         mel_abi_version(void);
/* Per-kernel timing of the last mel_step call, CUDA events on the handle's stream.
 * names: "contact", "body", "rigid", "proximity"; returns total milliseconds. */
mel_status  mel_get_kernel_times(mel_handle* h, double* ms_contact, double* ms_body,
                                 double* ms_rigid, double* ms_proximity, int* launches);
/* Device time of the last mel_step call (CUDA events around all of its launches), the
 * algorithmic bytes one launch of the body kernel and of the contact kernel moves (exact array
 * sizes of the resident layout), deformable node count and current contact count. */
mel_status  mel_get_step_stats(mel_handle* h, double* ms_total, double* bytes_body, double* bytes_contact,
                               int* n_deformable_nodes, int* n_contacts);
/* Launch configuration of the body kernel chosen at mel_create: support entries per chunk image,
 * dynamic shared memory per CTA (bytes) and CTAs per launch (one per body). */
mel_status  mel_get_kernel_config(mel_handle* h, int* chunk_cap, long long* body_smem, int* body_ctas);
/* Sizes of the resident model. */
mel_status  mel_get_sizes(mel_handle* h, int* n_bodies, int* n_nodes, int* n_gauss,
                          int* n_gp_entries, int* n_node_entries, int* n_border_nodes);

#ifdef __cplusplus
}
#endif
#endif /* MELGPU_H */
