// steps.h -- the per-model loop bodies and transform helpers, compiled in separate
// translation units (step_*.cu) and instantiated for float and double.
#pragma once

#include "ctx.cuh"

namespace smadft {

// no-adv/cosNoAdvTrackSing.cpp:681-764,1072 (keep_old: psi^{n+1} into S_PSI2)
template <typename T> int noadv_step(Ctx &c, bool keep_old);
// adv/cosAdvTrackMult.cpp:824-1369,1742
template <typename T> int adv_step(Ctx &c);
// the noadv / adv loop bodies of M batch members of one model and grid whose fields are
// pooled (member i's slot = mm[0]'s slot + i n elements), all on mm[0]'s stream; non-conserved
template <typename T> int noadv_group_step(Ctx *const *mm, int M);
template <typename T> int adv_group_step(Ctx *const *mm, int M);
// its first part (:847-1286): psi, grad psi, Sp2, S-hat and v from psihat into their slots
template <typename T> int adv_fields(Ctx &c);
// quasi/quasi.cpp:1099-2190 (nloop = 1-based step counter)
template <typename T> int quasi_step(Ctx &c, long long nloop, bool keep_old);
// compressible/compressible.cpp:1265-2720 (nloop = 1-based step counter); its pre-loop block
// (:1150-1194) and the mass / energy sums of a step (:2647-2690, psi_new = the step's psi)
template <typename T> int comp_step(Ctx &c, long long nloop, bool keep_old);
template <typename T> int comp_pre_loop(Ctx &c);
template <typename T> int reduce_comp_mass_energy(Ctx &c, const T *psi_new, double *ms);
// pre-loop blocks: no-adv :618-635, adv :760-777, quasi :990-1062
template <typename T> int pre_loop(Ctx &c);
// psi = REDFT01^3 psihat into dst
template <typename T> int refresh_psi(Ctx &c, T *dst);
// f' = REDFT01^3(alpha (q0^2 - q^2) psihat) into dst (quasi/quasi.cpp:1121-1137)
template <typename T> int dfd_field(Ctx &c, T *dst);
// psihat = scale REDFT10^3 psi (the reference's per-step planPsi, host-psi steps)
template <typename T> int psihat_from_psi(Ctx &c);
// plain transforms on caller buffers
template <typename T> int plain_r2r3d(Ctx &c, const T *in, T *out, int kx, int ky, int kz);
template <typename T> int plain_pass(Ctx &c, const T *in, T *out, int axis, int kind);
// quasi diagnostics sums: ms[0] = sum rho, ms[1] = sum e
template <typename T> int reduce_mass_energy(Ctx &c, double *ms);

// device scratch of smadft_step_surface (allocated on first use)
struct SurfaceScratch {
    double *psih_prev = nullptr;   // psihat^n (n doubles)
    void *fields = nullptr;        // dTpsi, psi_xx, psi_yy, psi_zz (4 n elements of the field type)
    int *idx = nullptr;            // per column: interface index along z (nx ny)
    double *vel = nullptr, *curvH = nullptr, *curvK = nullptr;
};
// one loop body with the interface diagnostics (surface.cu; noadv, adv)
template <typename T> int surface_step(Ctx &c, SurfaceScratch &sc);
// adjoint of `o.steps` noadv loop bodies from the initial condition (adjoint.cu)
template <typename T> int noadv_adjoint(Ctx &c, const smadft_adj_opts &o, smadft_grads *out, double *dpsi0_host);
// the same for the advected model (adjoint.cu)
template <typename T> int adv_adjoint(Ctx &c, const smadft_adj_opts &o, smadft_grads *out, double *dpsi0_host);

}  // namespace smadft
