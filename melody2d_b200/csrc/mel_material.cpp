// Body::Update_material's stiffness and damping updates (Code/Body.h:2708-2875) for mel_create.
//
// E and Nu come from the material as in Body.h:2727-2746 (other material types give 0, so the
// matrices become 0).  The elasticity matrix is the plane-strain one scaled by E/((1+Nu)(1-2Nu));
// per Gauss point, every entry of the local matrix of the support's dofs is summed from 0 in the
// reference's four-term order, and every upper-triangle dof pair adds L*weight*jacobian into the
// first MATRICES entry with those dofs (pairs without one are dropped).  The reference finds that
// entry by a linear search per pair; here a hash of the body's (dof0, dof1) pairs gives the same
// first index.  Each entry receives its terms Gauss point by Gauss point, as in the reference.
#include <cstdint>
#include <unordered_map>
#include <vector>
#include "mel_material.h"

void mel_set_error(const char* fmt, ...);

static void elastic_constants(const mel_model_desc* d, int mat, double& E, double& Nu)
{
    const double* P = d->material_params + MEL_MAT_NPARAM * mat;
    E = 0.; Nu = 0.;
    if (d->material_type[mat] == MEL_MAT_ELASTIC_LINEAR) {
        const double Mu = P[3], Lambda = P[4];
        E = Mu * (3. * Lambda + 2. * Mu) / (Lambda + Mu);
        Nu = Mu / (2. * Lambda + 2. * Mu);
    } else if (d->material_type[mat] == MEL_MAT_NEOHOOKEAN) {
        const double Mu = P[3], Kappa = P[4];
        E = 9. * Kappa * Mu / (3. * Kappa + Mu);
        Nu = (3. * Kappa - 2. * Mu) / (6. * Kappa + 2. * Mu);
    }
}

static mel_status assemble_body(const mel_model_desc* d, int b, double* mk)
{
    double E, Nu;
    elastic_constants(d, d->body_material[b], E, Nu);
    double C[3][3] = { { 1. - Nu, Nu, 0 }, { Nu, 1. - Nu, 0 }, { 0, 0, 1. - 2. * Nu } };
    for (auto& row : C)
        for (double& c : row) c *= E / ((1. + Nu) * (1. - 2. * Nu));
    const int nn = d->body_node_ptr[b + 1] - d->body_node_ptr[b];
    std::unordered_map<uint64_t, int> first;
    const int m0 = d->body_matrix_ptr[b], m1 = d->body_matrix_ptr[b + 1];
    first.reserve((size_t)(m1 - m0) * 2);
    for (int i = m1 - 1; i >= m0; i--) {
        mk[i] = 0.;
        first[(uint64_t)(uint32_t)d->matrix_dofs[2 * i] << 32 | (uint32_t)d->matrix_dofs[2 * i + 1]] = i;
    }
    std::vector<double> L;
    for (int g = d->body_gp_ptr[b]; g < d->body_gp_ptr[b + 1]; g++) {
        const int s0 = d->gp_sup_ptr[g], nin = d->gp_sup_ptr[g + 1] - s0, w = 2 * nin;
        const double* xd = d->gp_dNdx + s0;
        const double* yd = d->gp_dNdy + s0;
        for (int k = 0; k < nin; k++)
            if (d->gp_sup_idx[s0 + k] < 0 || d->gp_sup_idx[s0 + k] >= nn) {
                mel_set_error("Gauss point %d of body %d names node %d outside the body", g, b, d->gp_sup_idx[s0 + k]);
                return MEL_ERR_INVALID;
            }
        L.assign((size_t)w * w, 0.);
        for (int ii = 0; ii < nin; ii++)
            for (int jj = 0; jj < nin; jj++) {
                double* e = &L[(size_t)(2 * ii) * w + 2 * jj];                 // x row, x column
                *e += xd[ii] * C[0][0] * xd[jj]; *e += xd[ii] * C[0][2] * yd[jj];
                *e += yd[ii] * C[2][0] * xd[jj]; *e += yd[ii] * C[2][2] * yd[jj];
                e = &L[(size_t)(2 * ii) * w + 2 * jj + 1];                      // x row, y column
                *e += xd[ii] * C[0][1] * yd[jj]; *e += xd[ii] * C[0][2] * xd[jj];
                *e += yd[ii] * C[2][1] * yd[jj]; *e += yd[ii] * C[2][2] * xd[jj];
                e = &L[(size_t)(2 * ii + 1) * w + 2 * jj];                      // y row, x column
                *e += yd[ii] * C[1][0] * xd[jj]; *e += yd[ii] * C[1][2] * yd[jj];
                *e += xd[ii] * C[2][0] * xd[jj]; *e += xd[ii] * C[2][2] * yd[jj];
                e = &L[(size_t)(2 * ii + 1) * w + 2 * jj + 1];                  // y row, y column
                *e += yd[ii] * C[1][1] * yd[jj]; *e += yd[ii] * C[1][2] * xd[jj];
                *e += xd[ii] * C[2][1] * yd[jj]; *e += xd[ii] * C[2][2] * xd[jj];
            }
        for (int i = 0; i < w; i++) {
            const uint32_t dof0 = 2 * d->gp_sup_idx[s0 + i / 2] + (i & 1);
            for (int j = 0; j < w; j++) {
                const uint32_t dof1 = 2 * d->gp_sup_idx[s0 + j / 2] + (j & 1);
                if (dof1 < dof0) continue;
                auto it = first.find((uint64_t)dof0 << 32 | dof1);
                if (it != first.end()) mk[it->second] += L[(size_t)i * w + j] * d->gp_weight[g] * d->gp_jacobian[g];
            }
        }
    }
    return MEL_OK;
}

mel_status mel_update_matrices(const mel_model_desc* d, const double* node_mass, double* mk, double* mc)
{
    if (d->n_matrix <= 0 || (d->flags[5] != 1 && d->flags[6] != 1)) return MEL_OK;
    for (int b = 0; b < d->n_bodies; b++) {
        if (d->body_type[b] != MEL_BODY_DEFORMABLE) continue;
        if (d->flags[5] == 1) {
            mel_status st = assemble_body(d, b, mk);
            if (st != MEL_OK) return st;
        }
        if (d->flags[6] == 1) {
            const double* P = d->material_params + MEL_MAT_NPARAM * d->body_material[b];
            const double Alpha = P[1], Beta = P[2];
            const int n0 = d->body_node_ptr[b];
            for (int i = d->body_matrix_ptr[b]; i < d->body_matrix_ptr[b + 1]; i++) {
                const int d0 = d->matrix_dofs[2 * i], d1 = d->matrix_dofs[2 * i + 1];
                if (d0 == d1) mc[i] = Alpha * mk[i] + Beta * node_mass[2 * (n0 + d0 / 2)];
                else mc[i] = Alpha * mk[i];
            }
        }
    }
    return MEL_OK;
}
