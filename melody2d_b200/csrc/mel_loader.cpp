// Reader of the reference's input files.  It consumes tokens in the same order as Load_static
// (Code/IO.h:598-1861) and Load_dynamic (Code/IO.h:1871-2345) so that any file the reference
// accepts yields the same model; sections that only drive output (MONITORING, SPIES, GRAPHIC,
// DEACTIVATION definitions) are skipped line by line as the reference's outer loop would.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <map>
#include <sstream>
#include <string>
#include <vector>
#include "mel_host.h"

void mel_set_error(const char* fmt, ...);

void mel_host_model::finalize()
{
    mel_model_desc& d = desc;
    memset(&d, 0, sizeof d);
    d.abi_version = MELGPU_ABI_VERSION;
    auto I = [](std::vector<int>& v) -> const int* { if (v.empty()) v.push_back(0); return v.data(); };
    auto D = [](std::vector<double>& v) -> const double* { if (v.empty()) v.push_back(0.); return v.data(); };
    d.n_materials = (int)material_type.size();
    d.material_type = I(material_type); d.material_params = D(material_params);
    d.n_laws = (int)law_type.size();
    d.law_type = I(law_type); d.law_length = I(law_length); d.law_params = D(law_params); d.contacts_table = I(contacts_table);
    d.n_bodies = (int)body_type.size();
    d.body_type = I(body_type); d.body_material = I(body_material); d.body_periodic = I(body_periodic); d.body_status = I(body_status);
    d.body_dist = D(body_dist); d.body_node_ptr = I(body_node_ptr); d.body_border_ptr = I(body_border_ptr);
    d.body_gp_ptr = I(body_gp_ptr); d.body_cell_ptr = I(body_cell_ptr); d.rigid = D(rigid);
    d.n_nodes = (int)node_domain.size();
    d.node_x0 = D(node_x0); d.node_mass = D(node_mass); d.node_inv_mass = D(node_inv_mass); d.node_domain = D(node_domain);
    d.node_sup_ptr = I(node_sup_ptr); d.node_sup_idx = I(node_sup_idx); d.node_sup_N = D(node_sup_N); d.node_state = D(node_state);
    d.n_borders = (int)border_body.size();
    d.border_body = I(border_body); d.border_periodicity = I(border_periodicity); d.border_interpolant = I(border_interpolant);
    d.border_before = I(border_before); d.border_after = I(border_after); d.border_node_ptr = I(border_node_ptr);
    d.border_nodes = I(border_nodes); d.border_bc_type = I(border_bc_type); d.border_bc_param = D(border_bc_param);
    d.border_hist_ptr = I(border_hist_ptr); d.hist_time = D(hist_time); d.hist_value = D(hist_value);
    d.n_gauss = (int)gp_weight.size();
    d.gp_sup_ptr = I(gp_sup_ptr); d.gp_sup_idx = I(gp_sup_idx); d.gp_N = D(gp_N); d.gp_dNdx = D(gp_dNdx); d.gp_dNdy = D(gp_dNdy);
    d.gp_weight = D(gp_weight); d.gp_jacobian = D(gp_jacobian);
    d.n_cells = (int)(cells.size() / 3);
    d.cells = I(cells);
    d.n_matrix = (int)matrix_stiffness.size();
    d.body_matrix_ptr = I(body_matrix_ptr); d.matrix_dofs = I(matrix_dofs);
    d.matrix_stiffness = D(matrix_stiffness); d.matrix_damping = D(matrix_damping);
    deactivated_flat.assign(deactivated.size() * MEL_DEACT_NF, 0.);
    for (size_t i = 0; i < deactivated.size(); i++)
        for (size_t k = 0; k < deactivated[i].size() && k < MEL_DEACT_NF; k++) deactivated_flat[MEL_DEACT_NF * i + k] = deactivated[i][k];
    d.n_deactivated = (int)deactivated.size();
    d.deactivated = deactivated.empty() ? nullptr : deactivated_flat.data();
    if (!alid_time.empty()) {
        d.body_alid_ptr = body_alid_ptr.data();
        d.alid_time = alid_time.data(); d.alid_value = alid_value.data(); d.node_alid = node_alid.data();
    }
}

namespace {

struct BodyTmp {
    int type = 0, material = 0, periodic = 0, status = MEL_STATUS_ACTIVE;
    double dist[3] = { 0, 0, 0 };
    double rigid[MEL_RIGID_NF] = { 0 };
    // borders (control part)
    struct Bd {
        int per = 0, itp = 0, nbn = 0, before = 0, after = 0;
        int bc[2] = { MEL_BC_NONE, MEL_BC_NONE };
        double prm[4] = { 0, 0, 0, 0 };
        std::vector<double> ht[2], hv[2];
        std::vector<int> nodes;
    };
    std::vector<Bd> borders;
    // data part
    std::vector<double> x0, mass, imass, domain;
    std::vector<std::vector<int>> sup_idx;
    std::vector<std::vector<double>> sup_N;
    std::vector<double> gw, gJ;
    std::vector<std::vector<int>> gidx;
    std::vector<std::vector<double>> gN, gdx, gdy;
    int nregions = 1;
    std::vector<int> cells;
    std::vector<int> mdofs;
    std::vector<double> mk, mc;
    std::vector<double> state;   // 12 per node
    // ALID block (Code/IO.h:1395-1480): histories and the layer's geometry and grading
    std::vector<double> alid_t[2], alid_v[2];
    double alid[10] = { 0., 0., 0., 0., 0., 0., 0., 0., 0., 0. };   // xmin xmax ymin ymax range ain aout bin bout exponent
    std::vector<double> alid_ab;   // 2 per node
};

// alid_alpha, alid_beta of a node at (x, y) as Load_static computes them while reading NODES
// (Code/IO.h:1548-1600): graded layers along y, then along x keeping the larger value
void alid_node(const double* A, double x, double y, double* al, double* be)
{
    const double xmin = A[0], xmax = A[1], ymin = A[2], ymax = A[3], range = A[4];
    const double ain = A[5], aout = A[6], bin = A[7], bout = A[8], ex = A[9];
    double ka, kb, temp;
    *al = 0.; *be = 0.;
    if (y < ymin + range) {
        ka = (aout - ain) / pow(-range, ex);
        kb = (bout - bin) / pow(-range, ex);
        *al = ain + ka * pow(y - (ymin + range), ex);
        *be = bin + kb * pow(y - (ymin + range), ex);
    } else if (y > ymax - range) {
        ka = (aout - ain) / pow(range, ex);
        kb = (bout - bin) / pow(range, ex);
        *al = ain + ka * pow(y - (ymax - range), ex);
        *be = bin + kb * pow(y - (ymax - range), ex);
    }
    if (x < xmin + range) {
        ka = (aout - ain) / pow(-range, ex);
        kb = (bout - bin) / pow(-range, ex);
        temp = ain + ka * pow(x - (xmin + range), ex);
        if (temp > *al) *al = temp;
        temp = bin + kb * pow(x - (xmin + range), ex);
        if (temp > *be) *be = temp;
    } else if (x > xmax - range) {
        ka = (aout - ain) / pow(range, ex);
        kb = (bout - bin) / pow(range, ex);
        temp = ain + ka * pow(x - (xmax - range), ex);
        if (temp > *al) *al = temp;
        temp = bin + kb * pow(x - (xmax - range), ex);
        if (temp > *be) *be = temp;
    }
}

int per_code(const std::string& s) { return s == "Periodic" ? MEL_PER_PERIODIC : (s == "Simple" ? MEL_PER_SIMPLE : MEL_PER_CLOSED); }

const char* law_names[] = { "Frictionless", "Cohesion", "MohrCoulomb", "DampedMohrCoulomb", "TwoSlopesMohrCoulomb",
                            "BondedMohrCoulomb", "CZMlinear", "CZMfatigue" };
const int law_nparam[] = { 1, 4, 5, 6, 6, 11, 6, 9 };

// reads one direction's boundary condition block of a BORDERS section (Code/IO.h:1087-1176)
bool read_bc(std::istream& f, BodyTmp::Bd& br, int dir)
{
    std::string direction, type1, type2, token;
    f >> direction >> type1;
    if (type1 == "None") { br.bc[dir] = MEL_BC_NONE; std::getline(f, token); return true; }
    int nv = 0;
    if (type1 == "Dirichlet") {
        f >> type2;
        if (type2 == "Soft") { br.bc[dir] = MEL_BC_SOFT; f >> br.prm[2 * dir] >> br.prm[2 * dir + 1]; std::getline(f, token); }
        else if (type2 == "Driven") { br.bc[dir] = MEL_BC_DRIVEN; std::getline(f, token); }
    } else if (type1 == "Neumann") {
        f >> type2;
        if (type2 == "Oriented") br.bc[dir] = MEL_BC_ORIENTED;
        else if (type2 == "Following") br.bc[dir] = MEL_BC_FOLLOWING;
        std::getline(f, token);
    } else return false;
    f >> nv;
    std::getline(f, token);
    for (int j = 0; j < nv; j++) {
        double t, v;
        f >> t >> v;
        std::getline(f, token);
        br.ht[dir].push_back(t);
        br.hv[dir].push_back(v);
    }
    return true;
}

} // namespace

// One entry of a MONITORING (or SPIES / DEACTIVATION) list: the keyword grammar of Read_spy_line
// (Code/IO.h:11-590) and the vector it builds, {type, ...}.  Tables map each keyword to its code; the
// numbers that follow are read as the grammar says.  A keyword the grammar does not know leaves `v`
// as it was (the reference reuses the caller's vector the same way).
static void read_spy_line(std::istream& C, std::vector<double>& v)
{
    static const std::map<std::string, int> quantity = { { "Position", 0 }, { "Displacement", 1 }, { "Velocity", 2 },
                                                         { "Acceleration", 3 }, { "Force", 4 }, { "Jacobian", 5 },
                                                         { "Stress", 6 }, { "Contact", 7 }, { "Damage", 8 },
                                                         { "Energy", 9 }, { "Work", 10 }, { "Error", 11 },
                                                         { "MassScaling", 12 } };
    static const std::vector<std::string> position = { "X", "Y", "R", "Length", "LengthInContact", "Area", "AllX", "AllY" };
    static const std::vector<std::string> vector4 = { "X", "Y", "Mag", "R" };
    static const std::vector<std::string> forces = { "Total", "Internal", "Contact", "Body", "Dirichlet", "Neumann", "Damping", "Alid" };
    static const std::vector<std::string> stress = { "XX", "YY", "XY", "ZZ", "Tresca", "VM", "Major", "Intermediate", "Minor", "Spherical" };
    static const std::vector<std::string> contact = { "Gapn", "Gapt", "Xsi", "Xnorm", "Ynorm", "Damage", "Fx", "Fy", "Length",
                                                      "Master", "Px", "Py", "Slave", "Xslave", "Yslave" };
    static const std::vector<std::string> energy = { "Kinetic", "Deformation" };
    static const std::vector<std::string> work = { "Internal", "Contact", "Body", "Dirichlet", "Neumann", "Damping", "Alid" };
    static const std::vector<std::string> error = { "X", "Y", "Mag", "Norm", "Max" };
    static const std::vector<std::string> mass = { "X", "Y", "Moy", "dX", "dY", "dMoy", "Xmass", "Ymass", "Mass" };
    auto code = [](const std::vector<std::string>& t, const std::string& k) {
        for (size_t i = 0; i < t.size(); i++) if (t[i] == k) return (int)i;
        return -1;
    };
    std::string kw, sub;
    C >> kw;
    auto q = quantity.find(kw);
    if (q == quantity.end()) return;
    const double T = q->second;
    double b = 0, bo = 0, n = 0;
    int k;
    switch (q->second) {
    case 0:
        C >> sub;
        if ((k = code(position, sub)) < 0) return;
        if (k <= 2) { C >> b >> n; v = { T, (double)k, b, n }; }
        else if (k <= 5) { C >> b; v = { T, (double)k, b }; }
        else v = { T, (double)k };
        return;
    case 1: case 2: case 3:
        C >> sub;
        if ((k = code(vector4, sub)) < 0) return;
        C >> b >> n; v = { T, (double)k, b, n };
        return;
    case 4: {
        C >> sub;
        const int comp = code(vector4, sub);
        if (comp < 0) return;
        C >> sub;
        if ((k = code(forces, sub)) < 0) return;
        C >> b >> n; v = { T, (double)comp, (double)k, b, n };
        return;
    }
    case 5: case 8:
        if (q->second == 5) { C >> b >> n; v = { T, b, n }; }
        else { C >> b; v = { T, b }; }
        return;
    case 6:
        C >> sub;
        if ((k = code(stress, sub)) < 0) return;
        C >> b >> n; v = { T, (double)k, b, n };
        return;
    case 7:
        C >> sub;
        if ((k = code(contact, sub)) < 0) return;
        C >> b >> bo >> n; v = { T, (double)k, b, bo, n };
        return;
    case 9: case 10:
        C >> sub >> b;
        if ((k = code(q->second == 9 ? energy : work, sub)) < 0) return;
        v = { T, (double)k, b };
        return;
    case 11:
        C >> sub;
        if ((k = code(error, sub)) < 0) return;
        C >> b >> n; v = { T, (double)k, b, n };
        return;
    case 12:
        C >> sub;
        if (sub == "Polar") {
            double x0, x1, y0, y1;
            C >> sub >> n >> x0 >> x1 >> y0 >> y1;
            if (sub == "Contact_Normal") v = { 11., 0., n, x0, x1, y0, y1 };
            return;
        }
        if ((k = code(mass, sub)) < 0) return;
        C >> b >> n; v = { T, (double)k, b, n };
        return;
    }
}

mel_status mel_load_files(const char* dir, int restart_index, mel_host_model* out)
{
    mel_host_model& M = *out;
    std::string base = dir ? std::string(dir) : std::string(".");
    std::ifstream C(base + "/STATIC_CONTROL.asc");
    if (!C) { mel_set_error("cannot open %s/STATIC_CONTROL.asc", base.c_str()); return MEL_ERR_IO; }
    std::string line, token;
    int nmat = 0, nlaw = 0, nbodies = 0, index_body = 0;
    std::vector<std::string> law_m1, law_m2;
    std::vector<BodyTmp> B;
    std::string solver;
    double tini = 0, dt = 0, tend = 0, sp[8] = { 0 }, save = 0, print = 0, cup = 0, xmin = 0, xmax = 0, gx = 0, gy = 0;
    while (std::getline(C, line)) {
        if (line.compare(0, 15, "SIMULATION_NAME") == 0) { C >> M.name; std::getline(C, token); }
        if (line.compare(0, 9, "MATERIALS") == 0) {
            C >> nmat; std::getline(C, token); std::getline(C, token);
            for (int i = 0; i < nmat; i++) {
                std::string name, type;
                C >> name; std::getline(C, token);
                C >> type; std::getline(C, token);
                double p[6];
                C >> p[0] >> p[1] >> p[2] >> p[3] >> p[4] >> p[5]; std::getline(C, token);
                double mu = p[3] / (2. * (1. + p[4]));                      // Code/IO.h:678
                if (type == "ElasticLinear") {
                    M.material_type.push_back(MEL_MAT_ELASTIC_LINEAR);
                    double lam = p[3] * p[4] / ((1. + p[4]) * (1. - 2. * p[4]));
                    double q[6] = { p[0], p[1], p[2], mu, lam, p[5] };
                    M.material_params.insert(M.material_params.end(), q, q + 6);
                } else if (type == "NeoHookean") {
                    M.material_type.push_back(MEL_MAT_NEOHOOKEAN);
                    double kap = p[3] / (3. * (1. - 2. * p[4]));
                    double q[6] = { p[0], p[1], p[2], mu, kap, p[5] };
                    M.material_params.insert(M.material_params.end(), q, q + 6);
                } else { mel_set_error("material type %s is not supported", type.c_str()); return MEL_ERR_UNSUPPORTED; }
                M.material_names.push_back(name);
                std::getline(C, token);
            }
        }
        if (line.compare(0, 12, "CONTACT_LAWS") == 0) {
            C >> nlaw; std::getline(C, token); std::getline(C, token);
            for (int i = 0; i < nlaw; i++) {
                std::string m1, m2, type, le;
                C >> m1; std::getline(C, token);
                C >> m2; std::getline(C, token);
                C >> type; std::getline(C, token);
                C >> le; std::getline(C, token);
                int t = -1;
                for (int k = 0; k < 8; k++) if (type == law_names[k]) t = k;
                if (t < 0) { mel_set_error("contact law %s is not supported", type.c_str()); return MEL_ERR_UNSUPPORTED; }
                double p[MEL_LAW_NPARAM] = { 0 };
                for (int k = 0; k < law_nparam[t]; k++) C >> p[k];
                std::getline(C, token);
                M.law_type.push_back(t);
                M.law_length.push_back(le == "Evolutive" ? MEL_LENGTH_EVOLUTIVE : MEL_LENGTH_FIXED);
                M.law_params.insert(M.law_params.end(), p, p + MEL_LAW_NPARAM);
                law_m1.push_back(m1); law_m2.push_back(m2);
                std::getline(C, token);
            }
            // Contacts_Table (Code/IO.h:797-812)
            M.contacts_table.assign((size_t)nmat * nmat, -1);
            for (int i = 0; i < nlaw; i++) {
                int nn = 0, pp = 0;
                for (int n = 0; n < nmat; n++) if (M.material_names[n] == law_m1[i]) nn = n;
                for (int p = 0; p < nmat; p++) if (M.material_names[p] == law_m2[i]) pp = p;
                M.contacts_table[(size_t)nn * nmat + pp] = i;
                M.contacts_table[(size_t)pp * nmat + nn] = i;
            }
        }
        if (line.compare(0, 6, "SOLVER") == 0) {
            C >> solver; std::getline(C, token);
            if (solver == "Euler" || solver == "Adaptive_Euler") {
                C >> tini >> dt >> tend; std::getline(C, token);
                C >> sp[0] >> sp[1] >> sp[2]; std::getline(C, token);
                C >> save >> print >> cup; std::getline(C, token);
                sp[7] = 1 / sp[0];
            } else if (solver == "Euler_2") {
                C >> tini >> dt >> tend; std::getline(C, token);
                C >> save >> print >> cup; std::getline(C, token);
            } else if (solver == "Mass_Scaling" || solver == "Adaptive_Mass_Scaling") {
                C >> tini >> dt >> tend; std::getline(C, token);
                C >> sp[0] >> sp[1] >> sp[2]; std::getline(C, token);
                C >> sp[3] >> sp[4] >> sp[5] >> sp[6]; std::getline(C, token);
                C >> save >> print >> cup; std::getline(C, token);
                sp[7] = 1 / sp[0];
            }
        }
        if (line.compare(0, 19, "PERIODIC_BOUNDARIES") == 0) { C >> xmin >> xmax; std::getline(C, token); }
        if (line.compare(0, 17, "PENALTY_PARAMETER") == 0) { double p; C >> p; std::getline(C, token); }
        if (line.compare(0, 7, "GRAVITY") == 0) { C >> gx >> gy; std::getline(C, token); }
        if (line.compare(0, 8, "PLOTTING") == 0) { std::getline(C, token); std::getline(C, token); }
        if (line.compare(0, 12, "DEACTIVATION") == 0) {     // Code/IO.h:947-968; acted on by Update_status
            int n = 0;
            C >> n;
            std::getline(C, token);
            std::vector<double> entry;
            for (int i = 0; i < n; i++) {
                read_spy_line(C, entry);
                std::string kw;
                double threshold = 0.;
                C >> kw >> threshold;
                if (kw == "below") entry.push_back(0.);
                else if (kw == "equal") entry.push_back(1.);
                else if (kw == "above") entry.push_back(2.);
                entry.push_back(threshold);
                if (entry.size() > MEL_DEACT_NF) { mel_set_error("DEACTIVATION entry %d has %zu values", i, entry.size()); return MEL_ERR_UNSUPPORTED; }
                M.deactivated.push_back(entry);
                std::getline(C, token);
            }
        }
        if (line.compare(0, 10, "MONITORING") == 0) {        // Code/IO.h:933-945
            int n = 0;
            C >> n; std::getline(C, token);
            std::vector<double> entry;
            for (int i = 0; i < n; i++) {
                read_spy_line(C, entry);
                M.monitored.push_back(entry);
                std::getline(C, token);
            }
        }
        if (line.compare(0, 13, "NUMBER_BODIES") == 0) { C >> nbodies; std::getline(C, token); B.resize(nbodies); }
        if (line.compare(0, 10, "DEFORMABLE") == 0 || line.compare(0, 5, "RIGID") == 0) {
            bool rigid = line.compare(0, 5, "RIGID") == 0;
            C >> index_body; std::getline(C, token);
            std::string mat, per;
            C >> mat; std::getline(C, token);
            C >> per; std::getline(C, token);
            if (index_body < 0 || index_body >= (int)B.size()) { mel_set_error("body index %d out of range", index_body); return MEL_ERR_INVALID; }
            BodyTmp& b = B[index_body];
            C >> b.dist[0] >> b.dist[1] >> b.dist[2]; std::getline(C, token);
            b.type = rigid ? MEL_BODY_RIGID : MEL_BODY_DEFORMABLE;
            b.periodic = (per == "Periodic");
            b.material = 0;
            for (int i = 0; i < nmat; i++) if (M.material_names[i] == mat) { b.material = i; break; }
        }
        if (line.compare(0, 7, "BORDERS") == 0) {
            int nbd = 0;
            C >> nbd; std::getline(C, token); std::getline(C, token);
            BodyTmp& b = B[index_body];
            b.borders.resize(nbd);
            for (int i = 0; i < nbd; i++) {
                std::string per, itp;
                C >> per >> itp; std::getline(C, token);
                C >> b.borders[i].nbn; std::getline(C, token);
                b.borders[i].per = per_code(per);
                b.borders[i].itp = (itp == "Spline") ? MEL_INTERP_SPLINE : MEL_INTERP_LINEAR;
                if (!read_bc(C, b.borders[i], 0) || !read_bc(C, b.borders[i], 1)) { mel_set_error("malformed boundary condition in body %d", index_body); return MEL_ERR_INVALID; }
                std::getline(C, token);
            }
        }
        if (line.compare(0, 4, "ALID") == 0) {
            // counts and the twelve numbers, the rest of their line and one more line, the x history,
            // one separating line when both histories exist, the y history (Code/IO.h:1395-1480)
            if (index_body < 0 || index_body >= (int)B.size()) { mel_set_error("ALID before any body"); return MEL_ERR_INVALID; }
            BodyTmp& b = B[index_body];
            int nx = 0, ny = 0;
            C >> nx >> ny;
            for (int k = 0; k < 10; k++) C >> b.alid[k];
            if (!C || nx < 0 || ny < 0) { mel_set_error("malformed ALID block in body %d", index_body); return MEL_ERR_INVALID; }
            std::getline(C, token); std::getline(C, token);
            for (int dir = 0; dir < 2; dir++) {
                const int nv = dir ? ny : nx;
                if (dir == 1 && nx > 0 && ny > 0) std::getline(C, token);
                b.alid_t[dir].resize(nv); b.alid_v[dir].resize(nv);
                for (int j = 0; j < nv; j++) { C >> b.alid_t[dir][j] >> b.alid_v[dir][j]; std::getline(C, token); }
            }
        }
    }
    C.close();

    std::ifstream S(base + "/STATIC_DATA.asc");
    if (!S) { mel_set_error("cannot open %s/STATIC_DATA.asc", base.c_str()); return MEL_ERR_IO; }
    bool rigid = false;
    while (std::getline(S, line)) {
        if (line.compare(0, 10, "DEFORMABLE") == 0) { rigid = false; S >> index_body; std::getline(S, token); }
        if (line.compare(0, 5, "RIGID") == 0) {
            rigid = true;
            S >> index_body; std::getline(S, token);
            BodyTmp& b = B[index_body];
            S >> b.rigid[MEL_RG_X0] >> b.rigid[MEL_RG_Y0]; std::getline(S, token);
            S >> b.rigid[MEL_RG_MASS] >> b.rigid[MEL_RG_INERTIA] >> b.rigid[MEL_RG_INV_MASS] >> b.rigid[MEL_RG_INV_INERTIA]; std::getline(S, token);
            b.rigid[MEL_RG_R0] = 0.;
        }
        if (line.compare(0, 5, "NODES") == 0) {
            int nn = 0;
            S >> nn; std::getline(S, token); std::getline(S, token);
            BodyTmp& b = B[index_body];
            b.x0.resize(2 * nn); b.mass.assign(2 * nn, 0.); b.imass.assign(2 * nn, 0.); b.domain.assign(nn, 0.);
            b.sup_idx.assign(nn, {}); b.sup_N.assign(nn, {});
            for (int i = 0; i < nn; i++) {
                double j;
                if (!rigid) S >> j >> b.x0[2 * i] >> b.x0[2 * i + 1] >> b.domain[i] >> b.mass[2 * i] >> b.mass[2 * i + 1] >> b.imass[2 * i] >> b.imass[2 * i + 1];
                else S >> j >> b.x0[2 * i] >> b.x0[2 * i + 1];
                std::getline(S, token);
            }
            b.alid_ab.assign(2 * nn, 0.);
            if (!rigid && (!b.alid_t[0].empty() || !b.alid_t[1].empty()))
                for (int i = 0; i < nn; i++) alid_node(b.alid, b.x0[2 * i], b.x0[2 * i + 1], &b.alid_ab[2 * i], &b.alid_ab[2 * i + 1]);
        }
        if (line.compare(0, 7, "BORDERS") == 0) {
            int nbd = 0;
            S >> nbd; std::getline(S, token); std::getline(S, token);
            BodyTmp& b = B[index_body];
            if ((int)b.borders.size() < nbd) b.borders.resize(nbd);
            for (int i = 0; i < nbd; i++) {
                std::getline(S, token);
                int nbn, bef, aft;
                S >> nbn >> bef >> aft; std::getline(S, token);
                b.borders[i].before = bef; b.borders[i].after = aft;
                b.borders[i].nodes.resize(nbn);
                b.borders[i].nbn = nbn;
                for (int j = 0; j < nbn; j++) { S >> b.borders[i].nodes[j]; std::getline(S, token); }
                std::getline(S, token);
            }
        }
        if (line.compare(0, 11, "INTEGRATION") == 0) {
            std::string integration;
            std::getline(S, integration);
            BodyTmp& b = B[index_body];
            int ng = 0, nreg = 1;
            bool gauss = integration.compare(0, 5, "Gauss") == 0;
            bool nodal = integration.compare(0, 5, "Nodal") == 0;
            if (!gauss && !nodal) { mel_set_error("unknown integration type"); return MEL_ERR_INVALID; }
            S >> ng >> nreg; std::getline(S, token); std::getline(S, token);
            b.nregions = nreg;
            b.gw.resize(ng); b.gJ.resize(ng); b.gidx.assign(ng, {}); b.gN.assign(ng, {}); b.gdx.assign(ng, {}); b.gdy.assign(ng, {});
            for (int i = 0; i < ng; i++) {
                std::getline(S, token);
                double xg, yg;
                int ni = 0;
                if (gauss) { S >> xg >> yg >> b.gw[i] >> b.gJ[i]; }
                else { S >> xg >> yg >> b.gw[i]; b.gJ[i] = 1.; }
                std::getline(S, token);
                S >> ni; std::getline(S, token);
                for (int j = 0; j < ni; j++) {
                    int node, n1, n2;
                    double sf = 0., dx, dy;
                    if (gauss) S >> node >> n1 >> n2 >> sf >> dx >> dy;
                    else S >> node >> n1 >> n2 >> dx >> dy;
                    std::getline(S, token);
                    b.gidx[i].push_back(node); b.gN[i].push_back(sf); b.gdx[i].push_back(dx); b.gdy[i].push_back(dy);
                }
                std::getline(S, token);
            }
        }
        if (line.compare(0, 13, "TRIANGULATION") == 0) {
            int nc = 0;
            S >> nc; std::getline(S, token);
            BodyTmp& b = B[index_body];
            b.cells.resize(3 * nc);
            for (int i = 0; i < nc; i++) { int n0; S >> n0 >> b.cells[3 * i] >> b.cells[3 * i + 1] >> b.cells[3 * i + 2]; std::getline(S, token); }
            std::getline(S, token);
        }
        if (line.compare(0, 11, "DOF_TO_DISP") == 0) {
            BodyTmp& b = B[index_body];
            int nn = (int)b.domain.size();
            for (int i = 0; i < nn; i++) {
                std::getline(S, token); std::getline(S, token);
                int ni = 0;
                S >> ni; std::getline(S, token);
                for (int j = 0; j < ni; j++) {
                    int node; double ss, sx, sy;
                    S >> node >> ss >> sx >> sy; std::getline(S, token);
                    b.sup_idx[i].push_back(node); b.sup_N[i].push_back(ss);
                }
            }
        }
        if (line.compare(0, 8, "MATRICES") == 0) {
            int nm = 0;
            S >> nm; std::getline(S, token); std::getline(S, token);
            BodyTmp& b = B[index_body];
            for (int i = 0; i < nm; i++) {
                int n1, n2; double s, dd;
                S >> n1 >> n2 >> s >> dd; std::getline(S, token);
                b.mdofs.push_back(n1); b.mdofs.push_back(n2); b.mk.push_back(s); b.mc.push_back(dd);
            }
        }
    }
    S.close();

    // dynamic file (Code/IO.h:1885-1901 name pattern)
    char fname[64];
    snprintf(fname, sizeof fname, "DYNAMIC_%05d.asc", restart_index);
    std::ifstream Dy(base + "/" + fname);
    if (!Dy) { mel_set_error("cannot open %s/%s", base.c_str(), fname); return MEL_ERR_IO; }
    int flags[MEL_NFLAGS] = { 0 };
    double time = 0., next_cup = 0.;
    int nsave = 0, niter = 0, nprint = 0;
    double next_save = 0, next_print = 0;
    for (auto& b : B) b.state.assign(12 * (b.x0.size() / 2), 0.);
    std::vector<std::vector<mel_contact>> dyn_contacts(B.size());
    while (std::getline(Dy, line)) {
        const char* kw[] = { "KILL_VELOCITY", "MONITOR_ENERGY", "MONITOR_BOUNDARIES", "INITIALIZE_CZM", "UPDATE_MASS_MATRIX",
                             "UPDATE_STIFFNESS_MATRIX", "UPDATE_DAMPING_MATRIX", "NO_LOG", "NO_MONITORING", "NO_SELF_CONTACT", "RESET_WORK" };
        for (int k = 0; k < MEL_NFLAGS; k++) if (line.compare(0, strlen(kw[k]), kw[k]) == 0) flags[k] = 1;
        if (line.compare(0, 6, "SOLVER") == 0) {
            Dy >> solver; std::getline(Dy, token);
            Dy >> nsave >> niter >> time >> nprint; std::getline(Dy, token);
            Dy >> dt; std::getline(Dy, token);
            Dy >> next_save >> next_print >> next_cup; std::getline(Dy, token);
        }
        if (line.compare(0, 10, "DEFORMABLE") == 0 || line.compare(0, 5, "RIGID") == 0) {
            rigid = line.compare(0, 5, "RIGID") == 0;
            std::string status;
            Dy >> status; std::getline(Dy, token);
            Dy >> index_body; std::getline(Dy, token);
            B[index_body].status = status == "inactive" ? MEL_STATUS_INACTIVE : (status == "nogravity" ? MEL_STATUS_NOGRAVITY : MEL_STATUS_ACTIVE);
        }
        if (line.compare(0, 10, "KINEMATICS") == 0) {
            BodyTmp& b = B[index_body];
            if (!rigid) {
                int nn = 0;
                Dy >> nn; std::getline(Dy, token);
                for (int i = 0; i < nn; i++) {
                    double j, xc, yc, v[12];
                    Dy >> j >> xc >> yc;
                    for (int k = 0; k < 12; k++) Dy >> v[k];
                    std::getline(Dy, token);
                    double* s = &b.state[12 * (size_t)i];
                    // file order: disp, vel, acc, disp param, vel param, acc param
                    for (int k = 0; k < 12; k++) s[k] = v[k];
                    if (flags[0] == 1) { s[2] = s[3] = 0.; s[8] = s[9] = 0.; }
                }
            } else {
                double xc, yc, rc, xd, yd, rd, xv, yv, rv;
                Dy >> xc >> yc >> rc; std::getline(Dy, token);
                Dy >> xd >> yd >> rd; std::getline(Dy, token);
                Dy >> xv >> yv >> rv; std::getline(Dy, token);
                b.rigid[MEL_RG_XD] = xd; b.rigid[MEL_RG_YD] = yd; b.rigid[MEL_RG_RD] = rd;
                if (flags[0] == 0) { b.rigid[MEL_RG_XV] = xv; b.rigid[MEL_RG_YV] = yv; b.rigid[MEL_RG_RV] = rv; }
            }
        }
        if (line.compare(0, 8, "CONTACTS") == 0) {
            int nc = 0;
            Dy >> nc; std::getline(Dy, token);
            for (int i = 0; i < nc; i++) {
                mel_contact c;
                memset(&c, 0, sizeof c);
                int ni = 0;
                Dy >> c.borderS >> c.border_nodeS >> c.nodeS >> c.bodyM >> c.borderM >> c.shiftM >> c.segmentM >> c.gapn >> c.gapt >> c.xsi;
                Dy >> c.xnorm >> c.ynorm >> c.xtan >> c.ytan;
                Dy >> c.length >> c.fx >> c.fy;
                for (int k = 0; k < 4; k++) Dy >> c.nodeM[k] >> c.shapeM[k] >> c.shiftMk[k];
                Dy >> c.effective_mass >> ni;
                for (int k = 0; k < ni; k++) { double v; Dy >> v; if (k < MEL_NINTERNAL) c.internal[k] = v; }
                c.nb_internal = ni;
                c.bodyS = index_body;
                dyn_contacts[index_body].push_back(c);
            }
        }
    }
    Dy.close();
    // flatten
    int nb = (int)B.size();
    M.body_node_ptr.push_back(0); M.body_border_ptr.push_back(0); M.body_gp_ptr.push_back(0); M.body_cell_ptr.push_back(0);
    M.body_matrix_ptr.push_back(0);
    M.node_sup_ptr.push_back(0); M.gp_sup_ptr.push_back(0); M.border_node_ptr.push_back(0); M.border_hist_ptr.push_back(0);
    for (int bi = 0; bi < nb; bi++) {
        BodyTmp& b = B[bi];
        int nn = (int)b.x0.size() / 2;
        M.body_type.push_back(b.type); M.body_material.push_back(b.material); M.body_periodic.push_back(b.periodic);
        M.body_status.push_back(b.status);
        M.body_dist.insert(M.body_dist.end(), b.dist, b.dist + 3);
        M.rigid.insert(M.rigid.end(), b.rigid, b.rigid + MEL_RIGID_NF);
        M.node_x0.insert(M.node_x0.end(), b.x0.begin(), b.x0.end());
        M.node_mass.insert(M.node_mass.end(), b.mass.begin(), b.mass.end());
        M.node_inv_mass.insert(M.node_inv_mass.end(), b.imass.begin(), b.imass.end());
        M.node_domain.insert(M.node_domain.end(), b.domain.begin(), b.domain.end());
        M.node_state.insert(M.node_state.end(), b.state.begin(), b.state.end());
        for (int i = 0; i < nn; i++) {
            for (size_t k = 0; k < b.sup_idx[i].size(); k++) { M.node_sup_idx.push_back(b.sup_idx[i][k]); M.node_sup_N.push_back(b.sup_N[i][k]); }
            M.node_sup_ptr.push_back((int)M.node_sup_idx.size());
        }
        M.body_node_ptr.push_back(M.body_node_ptr.back() + nn);
        for (auto& br : b.borders) {
            M.border_body.push_back(bi); M.border_periodicity.push_back(br.per); M.border_interpolant.push_back(br.itp);
            M.border_before.push_back(br.before); M.border_after.push_back(br.after);
            M.border_nodes.insert(M.border_nodes.end(), br.nodes.begin(), br.nodes.end());
            M.border_node_ptr.push_back((int)M.border_nodes.size());
            for (int dir = 0; dir < 2; dir++) {
                M.border_bc_type.push_back(br.bc[dir]);
                M.hist_time.insert(M.hist_time.end(), br.ht[dir].begin(), br.ht[dir].end());
                M.hist_value.insert(M.hist_value.end(), br.hv[dir].begin(), br.hv[dir].end());
                M.border_hist_ptr.push_back((int)M.hist_time.size());
            }
            M.border_bc_param.insert(M.border_bc_param.end(), br.prm, br.prm + 4);
        }
        M.body_border_ptr.push_back((int)M.border_body.size());
        for (size_t g = 0; g < b.gw.size(); g++) {
            for (size_t k = 0; k < b.gidx[g].size(); k++) {
                M.gp_sup_idx.push_back(b.gidx[g][k]); M.gp_N.push_back(b.gN[g][k]); M.gp_dNdx.push_back(b.gdx[g][k]); M.gp_dNdy.push_back(b.gdy[g][k]);
            }
            M.gp_sup_ptr.push_back((int)M.gp_sup_idx.size());
            M.gp_weight.push_back(b.gw[g]); M.gp_jacobian.push_back(b.gJ[g]);
        }
        M.body_gp_ptr.push_back((int)M.gp_weight.size());
        M.n_regions.push_back(b.nregions);
        M.cells.insert(M.cells.end(), b.cells.begin(), b.cells.end());
        M.body_cell_ptr.push_back((int)(M.cells.size() / 3));
        M.matrix_dofs.insert(M.matrix_dofs.end(), b.mdofs.begin(), b.mdofs.end());
        M.matrix_stiffness.insert(M.matrix_stiffness.end(), b.mk.begin(), b.mk.end());
        M.matrix_damping.insert(M.matrix_damping.end(), b.mc.begin(), b.mc.end());
        M.body_matrix_ptr.push_back((int)M.matrix_stiffness.size());
        for (auto& c : dyn_contacts[bi]) M.contacts.push_back(c);
    }
    // ALID layers: histories per (body, direction) and the nodal coefficients, when any body has one
    bool any_alid = false;
    for (auto& b : B) any_alid = any_alid || !b.alid_t[0].empty() || !b.alid_t[1].empty();
    if (any_alid) {
        M.body_alid_ptr.push_back(0);
        for (auto& b : B) {
            for (int dir = 0; dir < 2; dir++) {
                M.alid_time.insert(M.alid_time.end(), b.alid_t[dir].begin(), b.alid_t[dir].end());
                M.alid_value.insert(M.alid_value.end(), b.alid_v[dir].begin(), b.alid_v[dir].end());
                M.body_alid_ptr.push_back((int)M.alid_time.size());
            }
            if (b.alid_ab.size() == b.x0.size()) M.node_alid.insert(M.node_alid.end(), b.alid_ab.begin(), b.alid_ab.end());
            else M.node_alid.insert(M.node_alid.end(), b.x0.size(), 0.);
        }
    }
    mel_model_desc& d = M.desc;
    M.finalize();
    d.period[0] = xmin; d.period[1] = xmax;
    d.gravity[0] = gx; d.gravity[1] = gy;
    d.time = time; d.dt = dt; d.tend = tend;
    d.contact_update_period = cup; d.next_contact_update = next_cup;
    const char* sn[] = { "Euler", "Adaptive_Euler", "Mass_Scaling", "Adaptive_Mass_Scaling", "Euler_2" };
    d.solver = -1;
    for (int k = 0; k < 5; k++) if (solver == sn[k]) d.solver = k;
    if (d.solver < 0) { mel_set_error("unknown solver %s", solver.c_str()); return MEL_ERR_INVALID; }
    for (int k = 0; k < 8; k++) d.solver_params[k] = sp[k];
    for (int k = 0; k < MEL_NFLAGS; k++) d.flags[k] = flags[k];
    (void)tini;
    M.save_period = save; M.print_period = print;
    M.number_save = nsave; M.number_iteration = niter; M.number_print = nprint;
    M.next_save = next_save; M.next_print = next_print;
    return MEL_OK;
}
