// step_adv.cu -- the advected loop body (adv/cosAdvTrackMult.cpp:824-1369,1742).
#include "models.cuh"
#include "steps.h"

namespace smadft {

template <typename T>
int adv_step(Ctx &c)
{
    Spec<T> s = make_spec<T>(c);
    T *psi = c.f<T>(S_PSI), *ph = c.f<T>(S_PSIH), *np = c.f<T>(S_NP);
    T *gx = c.f<T>(S_GX), *gy = c.f<T>(S_GY), *gz = c.f<T>(S_GZ), *sp2 = c.f<T>(S_SP2);
    T *Sx = c.f<T>(S_SX), *Sy = c.f<T>(S_SY), *Sz = c.f<T>(S_SZ);
    T *vx = c.f<T>(S_VX), *vy = c.f<T>(S_VY), *vz = c.f<T>(S_VZ);
    int rc;
    // psi and grad psi from psihat (adv/cosAdvTrackMult.cpp:904-975)
    if ((rc = r2r3d<T>(c, K_DCT3, K_DCT3, K_DCT3, LoadArr<T>{ph}, StoreArr<T>{psi}))) return rc;
    if ((rc = r2r3d<T>(c, K_DST3, K_DCT3, K_DCT3, LdGrad<T, 0>{s, ph}, StoreArr<T>{gx}))) return rc;
    if ((rc = r2r3d<T>(c, K_DCT3, K_DST3, K_DCT3, LdGrad<T, 1>{s, ph}, StoreArr<T>{gy}))) return rc;
    if ((rc = r2r3d<T>(c, K_DCT3, K_DCT3, K_DST3, LdGrad<T, 2>{s, ph}, StoreArr<T>{gz}))) return rc;
    // Sp2 = iCT(-L psihat) (:980-991)
    if ((rc = r2r3d<T>(c, K_DCT3, K_DCT3, K_DCT3, LdNegLin<T>{s, ph}, StoreArr<T>{sp2}))) return rc;
    // force spectra S_c = ST_c(mu d_c psi) (:996-1027)
    if ((rc = r2r3d<T>(c, K_DST2, K_DCT2, K_DCT2, LdForce<T>{psi, sp2, gx, s.beta, s.gamma}, StoreArr<T>{Sx}))) return rc;
    if ((rc = r2r3d<T>(c, K_DCT2, K_DST2, K_DCT2, LdForce<T>{psi, sp2, gy, s.beta, s.gamma}, StoreArr<T>{Sy}))) return rc;
    if ((rc = r2r3d<T>(c, K_DCT2, K_DCT2, K_DST2, LdForce<T>{psi, sp2, gz, s.beta, s.gamma}, StoreArr<T>{Sz}))) return rc;
    // Stokes velocity (:1030-1286)
    if ((rc = r2r3d<T>(c, K_DST3, K_DCT3, K_DCT3, LdStokes<T, 0, false>{s, Sx, Sy, Sz, nullptr}, StoreArr<T>{vx}))) return rc;
    if ((rc = r2r3d<T>(c, K_DCT3, K_DST3, K_DCT3, LdStokes<T, 1, false>{s, Sx, Sy, Sz, nullptr}, StoreArr<T>{vy}))) return rc;
    if ((rc = r2r3d<T>(c, K_DCT3, K_DCT3, K_DST3, LdStokes<T, 2, false>{s, Sx, Sy, Sz, nullptr}, StoreArr<T>{vz}))) return rc;
    // N = beta psi^3 - gamma psi^5 - v.grad psi, CN/AB2 update (:1290-1365)
    return r2r3d<T>(c, K_DCT2, K_DCT2, K_DCT2,
                    LdAdvN<T>{psi, vx, vy, vz, gx, gy, gz, s.beta, s.gamma}, StUpdCN<T>{s, ph, np});
}

template int adv_step<float>(Ctx &);
template int adv_step<double>(Ctx &);

}  // namespace smadft
