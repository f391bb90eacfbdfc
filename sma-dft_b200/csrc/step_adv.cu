// step_adv.cu -- the advected loop body (adv/cosAdvTrackMult.cpp:824-1369,1742).
#include "models.cuh"
#include "steps.h"

namespace smadft {

// psi, grad psi and Sp2 = iCT(-L psihat) from psihat with the passes the gradients share with
// psi.  The gradient spectra are index-shifted, scaled copies of psihat along one axis
// (LdGrad), and shifting or scaling along one axis commutes with the transforms along the
// others.  So psi's y pass output P = iCT_y(psihat) also gives gz = iCT_x iST_z (LdGrad_z P),
// and psi's y + z output U = iCT_z P gives gx = iST_x (LdGrad_x U): the y passes of gx and gz
// and the z pass of gx are not run (12 axis passes instead of 15).  The order of operations
// differs from the reference's (scale, then transform) only in rounding.
template <typename T>
int adv_psi_fields_shared(Ctx &c, const Spec<T> &s, const double *ph, T *psi, T *gx, T *gy, T *gz, T *sp2)
{
    const int ky[3] = {K_DCT3, K_DST3, K_DCT3};
    T *const out[3] = {psi, gy, sp2};
    int rc = y_pass_multi<T, 3, 0>(c, ky, out, LoadArr<T, double>{ph}, LdGrad<T, 1, double>{s, ph}, LdNegLin<T>{s, ph});
    if (rc) return rc;
    // gz's z pass reads P before psi's z pass replaces it
    if ((rc = z_pass_grad<T>(c, s, psi, gz))) return rc;
    return forked(c, 4, [&](int m) {
        int r;
        switch (m) {
        case 0:   // psi: z pass, then gx's x pass reads U before psi's x pass replaces it
            if ((r = launch_axis<T, 2>(c, K_DCT3, LoadArr<T>{psi}, StoreArr<T>{psi}))) return r;
            if ((r = launch_axis<T, 0>(c, K_DST3, LdGrad<T, 0, T>{s, psi}, StoreArr<T>{gx}))) return r;
            return launch_axis<T, 0>(c, K_DCT3, LoadArr<T>{psi}, StoreArr<T>{psi});
        case 1: return launch_axis<T, 0>(c, K_DCT3, LoadArr<T>{gz}, StoreArr<T>{gz});
        default: {
            T *f = m == 2 ? gy : sp2;
            if ((r = launch_axis<T, 2>(c, K_DCT3, LoadArr<T>{f}, StoreArr<T>{f}))) return r;
            return launch_axis<T, 0>(c, K_DCT3, LoadArr<T>{f}, StoreArr<T>{f});
        }
        }
    });
}

// The force spectra stored by true wavenumber, then the Stokes velocity from them (LdStokesK):
// the sine-axis pass of each force component stores one index up along its axis (Sy in the
// grouped y pass, Sz in its z pass, Sx in its x pass); the projection then reads the three
// spectra of one wavenumber at one index, and v_z's sine z pass reads it one index up.  The
// values and operations are those of the reference's indexing; only where they are stored
// differs.  Needs the register-direct kernels on all three lengths.
template <typename T>
int adv_force_stokes_true_k(Ctx &c, const Spec<T> &s, T *psi, T *sp2, T *gx, T *gy, T *gz, T *Sx, T *Sy, T *Sz,
                            T *vx, T *vy, T *vz)
{
    int rc;
    {
        const KindSet<3> ks{{K_DCT2, K_DST2, K_DCT2}};
        const auto lm = make_multi(LdForce<T>{psi, sp2, gx, s.beta, s.gamma}, LdForce<T>{psi, sp2, gy, s.beta, s.gamma},
                                   LdForce<T>{psi, sp2, gz, s.beta, s.gamma});
        const StoreMultiUp<T, 3, 1> sm{{Sx, Sy, Sz}, 2u, (idx_t)c.g.nz, c.g.ny};
        using LM = std::remove_const_t<decltype(lm)>;
        using SM = StoreMultiUp<T, 3, 1>;
        switch (c.g.ny) {
        case 64: rc = launch_rd<T, 64, 1, LM, SM, 3, 1>(c, ks, lm, sm); break;
        case 128: rc = launch_rd<T, 128, 1, LM, SM, 3, 1>(c, ks, lm, sm); break;
        default: rc = launch_rd<T, 256, 1, LM, SM, 3, 1>(c, ks, lm, sm); break;
        }
        if (rc) return rc;
        rc = forked(c, 3, [&](int m) {
            int r;
            switch (m) {
            case 0:
                if ((r = launch_axis<T, 2>(c, K_DCT2, LoadArr<T>{Sx}, StoreArr<T>{Sx}))) return r;
                return launch_axis<T, 0>(c, K_DST2, LoadArr<T>{Sx}, StoreUp<T, 0>{Sx, (idx_t)c.g.nyz, c.g.nx});
            case 1:
                if ((r = launch_axis<T, 2>(c, K_DCT2, LoadArr<T>{Sy}, StoreArr<T>{Sy}))) return r;
                return launch_axis<T, 0>(c, K_DCT2, LoadArr<T>{Sy}, StoreArr<T>{Sy});
            default:
                if ((r = z_pass_upstore<T>(c, Sz, Sz))) return r;
                return launch_axis<T, 0>(c, K_DCT2, LoadArr<T>{Sz}, StoreArr<T>{Sz});
            }
        });
        if (rc) return rc;
    }
    const int ky[3] = {K_DCT3, K_DST3, K_DCT3};
    T *const out[3] = {vx, vy, vz};
    if ((rc = y_pass_multi<T, 3, 0>(c, ky, out, LdStokesK<T, 0>{s, Sx, Sy, Sz}, LdStokesK<T, 1>{s, Sx, Sy, Sz},
                                    LdStokesK<T, 2>{s, Sx, Sy, Sz})))
        return rc;
    return forked(c, 3, [&](int m) {
        int r;
        switch (m) {
        case 0:
            if ((r = launch_axis<T, 2>(c, K_DCT3, LoadArr<T>{vx}, StoreArr<T>{vx}))) return r;
            return launch_axis<T, 0>(c, K_DST3, LoadArr<T>{vx}, StoreArr<T>{vx});
        case 1:
            if ((r = launch_axis<T, 2>(c, K_DCT3, LoadArr<T>{vy}, StoreArr<T>{vy}))) return r;
            return launch_axis<T, 0>(c, K_DCT3, LoadArr<T>{vy}, StoreArr<T>{vy});
        default:
            if ((r = z_pass_upread<T>(c, vz, vz))) return r;
            return launch_axis<T, 0>(c, K_DCT3, LoadArr<T>{vz}, StoreArr<T>{vz});
        }
    });
}

inline bool rd_len(int n) { return n == 64 || n == 128 || n == 256; }

// psi, grad psi, Sp2, the force spectra S-hat and the velocity v of the current psihat: the
// loop body up to N (adv/cosAdvTrackMult.cpp:847-1286)
template <typename T>
int adv_fields(Ctx &c)
{
    Spec<T> s = make_spec<T>(c);
    T *psi = c.f<T>(S_PSI);
    double *ph = c.f<double>(S_PSIH);   // spectral state (FP64)
    T *gx = c.f<T>(S_GX), *gy = c.f<T>(S_GY), *gz = c.f<T>(S_GZ), *sp2 = c.f<T>(S_SP2);
    T *Sx = c.f<T>(S_SX), *Sy = c.f<T>(S_SY), *Sz = c.f<T>(S_SZ);
    T *vx = c.f<T>(S_VX), *vy = c.f<T>(S_VY), *vz = c.f<T>(S_VZ);
    int rc;
    // psi, grad psi and Sp2 = iCT(-L psihat), all from psihat (adv/cosAdvTrackMult.cpp:904-991)
    if (c.share_grad && c.use_rd && c.use_multi && !plane_ok(c) && (c.g.ny == 64 || c.g.ny == 128 || c.g.ny == 256)) {
        if ((rc = adv_psi_fields_shared<T>(c, s, ph, psi, gx, gy, gz, sp2))) return rc;
    } else {
        const int kx[5] = {K_DCT3, K_DST3, K_DCT3, K_DCT3, K_DCT3};
        const int ky[5] = {K_DCT3, K_DCT3, K_DST3, K_DCT3, K_DCT3};
        const int kz[5] = {K_DCT3, K_DCT3, K_DCT3, K_DST3, K_DCT3};
        T *const out[5] = {psi, gx, gy, gz, sp2};
        if ((rc = r2r3d_multi<T, 5, 0>(c, kx, ky, kz, out, LoadArr<T, double>{ph}, LdGrad<T, 0, double>{s, ph},
                                    LdGrad<T, 1, double>{s, ph}, LdGrad<T, 2, double>{s, ph}, LdNegLin<T>{s, ph})))
            return rc;
    }
    // force spectra S_c = ST_c(mu d_c psi) (:996-1027) and the Stokes velocity (:1030-1286)
    if (c.stokes_true_k && c.use_rd && c.use_rdz && c.use_multi && !plane_ok(c) && rd_len(c.g.nx) &&
        rd_len(c.g.ny) && rd_len(c.g.nz))
        return adv_force_stokes_true_k<T>(c, s, psi, sp2, gx, gy, gz, Sx, Sy, Sz, vx, vy, vz);
    {
        const int kx[3] = {K_DST2, K_DCT2, K_DCT2};
        const int ky[3] = {K_DCT2, K_DST2, K_DCT2};
        const int kz[3] = {K_DCT2, K_DCT2, K_DST2};
        T *const out[3] = {Sx, Sy, Sz};
        if ((rc = r2r3d_multi<T, 3, 1>(c, kx, ky, kz, out, LdForce<T>{psi, sp2, gx, s.beta, s.gamma},
                                    LdForce<T>{psi, sp2, gy, s.beta, s.gamma},
                                    LdForce<T>{psi, sp2, gz, s.beta, s.gamma})))
            return rc;
    }
    // Stokes velocity (:1030-1286)
    {
        const int kx[3] = {K_DST3, K_DCT3, K_DCT3};
        const int ky[3] = {K_DCT3, K_DST3, K_DCT3};
        const int kz[3] = {K_DCT3, K_DCT3, K_DST3};
        T *const out[3] = {vx, vy, vz};
        if ((rc = r2r3d_multi<T, 3, 0>(c, kx, ky, kz, out, LdStokes<T, 0, false>{s, Sx, Sy, Sz, nullptr},
                                    LdStokes<T, 1, false>{s, Sx, Sy, Sz, nullptr},
                                    LdStokes<T, 2, false>{s, Sx, Sy, Sz, nullptr})))
            return rc;
    }
    return SMADFT_OK;
}

template <typename T>
int adv_step(Ctx &c)
{
    int rc = adv_fields<T>(c);
    if (rc) return rc;
    Spec<T> s = make_spec<T>(c);
    T *psi = c.f<T>(S_PSI);
    double *ph = c.f<double>(S_PSIH);
    T *np = c.f<T>(S_NP);
    T *gx = c.f<T>(S_GX), *gy = c.f<T>(S_GY), *gz = c.f<T>(S_GZ);
    T *Sx = c.f<T>(S_SX);
    T *vx = c.f<T>(S_VX), *vy = c.f<T>(S_VY), *vz = c.f<T>(S_VZ);
    if (c.p.conserved) {
        // conserved: N = q^2 REDFT10^3(beta psi^3 - gamma psi^5) - REDFT10^3(v.grad psi)
        // (adv/cosAdvConSingle.cpp:1296-1310,1369); Sx is free once the velocity is out
        if ((rc = r2r3d<T>(c, K_DCT2, K_DCT2, K_DCT2, LdAdvDot<T>{vx, vy, vz, gx, gy, gz}, StoreArr<T>{Sx})))
            return rc;
        return r2r3d<T>(c, K_DCT2, K_DCT2, K_DCT2, LdNonlin<T>{psi, s.beta, s.gamma},
                        StUpdCN<T, 2>{make_spec<double>(c), ph, np, Sx});
    }
    // N = beta psi^3 - gamma psi^5 - v.grad psi, CN/AB2 update (:1290-1365)
    return r2r3d<T>(c, K_DCT2, K_DCT2, K_DCT2,
                    LdAdvN<T>{psi, vx, vy, vz, gx, gy, gz, s.beta, s.gamma}, StUpdCN<T>{make_spec<double>(c), ph, np});
}

// The same loop body for M batch members of one grid whose fields are pooled (member i's
// slot = the lead's slot + i n elements): per transform, the y passes with each member's
// loaders (its own parameters) run per member; the plain z and x passes run once over the
// pool; the CN/AB2 x pass runs per member (its storer carries the member's parameters).  All
// launches go to the lead's stream.  Non-conserved runs only.
template <typename T>
int adv_group_step(Ctx *const *mm, int M)
{
    Ctx &L = *mm[0];
    int rc;
    auto pz = [&](int slot, int kind) { return pooled_pass<T, 2>(L, M, kind, L.f<T>(slot), L.f<T>(slot)); };
    auto px = [&](int slot, int kind) { return pooled_pass<T, 0>(L, M, kind, L.f<T>(slot), L.f<T>(slot)); };
    // psi, grad psi and Sp2 from psihat (adv/cosAdvTrackMult.cpp:904-991)
    if (L.share_grad && L.use_rd && L.use_multi && (L.g.ny == 64 || L.g.ny == 128 || L.g.ny == 256)) {
        // the shared-pass order of adv_psi_fields_shared: the passes that carry a member's
        // wavenumbers (gz's z pass, gx's x pass) run per member, the plain ones over the pool
        const int ky[3] = {K_DCT3, K_DST3, K_DCT3};
        for (int i = 0; i < M; i++) {
            rc = on_lead_stream(L, *mm[i], [&](Ctx &c) {
                Spec<T> s = make_spec<T>(c);
                double *ph = c.f<double>(S_PSIH);
                T *const out[3] = {c.f<T>(S_PSI), c.f<T>(S_GY), c.f<T>(S_SP2)};
                const int r = y_pass_multi<T, 3, 0>(c, ky, out, LoadArr<T, double>{ph}, LdGrad<T, 1, double>{s, ph},
                                                    LdNegLin<T>{s, ph});
                return r ? r : z_pass_grad<T>(c, s, c.f<T>(S_PSI), c.f<T>(S_GZ));
            });
            if (rc) return rc;
        }
        if ((rc = pz(S_PSI, K_DCT3))) return rc;
        for (int i = 0; i < M; i++) {
            rc = on_lead_stream(L, *mm[i], [&](Ctx &c) {
                return launch_axis<T, 0>(c, K_DST3, LdGrad<T, 0, T>{make_spec<T>(c), c.f<T>(S_PSI)},
                                         StoreArr<T>{c.f<T>(S_GX)});
            });
            if (rc) return rc;
        }
        if ((rc = px(S_PSI, K_DCT3)) || (rc = px(S_GZ, K_DCT3))) return rc;
        for (int slot : {S_GY, S_SP2})
            if ((rc = pz(slot, K_DCT3)) || (rc = px(slot, K_DCT3))) return rc;
    } else {
        const int kx[5] = {K_DCT3, K_DST3, K_DCT3, K_DCT3, K_DCT3};
        const int ky[5] = {K_DCT3, K_DCT3, K_DST3, K_DCT3, K_DCT3};
        const int kz[5] = {K_DCT3, K_DCT3, K_DCT3, K_DST3, K_DCT3};
        const int slots[5] = {S_PSI, S_GX, S_GY, S_GZ, S_SP2};
        for (int i = 0; i < M; i++) {
            rc = on_lead_stream(L, *mm[i], [&](Ctx &c) {
                Spec<T> s = make_spec<T>(c);
                double *ph = c.f<double>(S_PSIH);
                T *const out[5] = {c.f<T>(S_PSI), c.f<T>(S_GX), c.f<T>(S_GY), c.f<T>(S_GZ), c.f<T>(S_SP2)};
                return y_pass_multi<T, 5, 0>(c, ky, out, LoadArr<T, double>{ph}, LdGrad<T, 0, double>{s, ph},
                                             LdGrad<T, 1, double>{s, ph}, LdGrad<T, 2, double>{s, ph},
                                             LdNegLin<T>{s, ph});
            });
            if (rc) return rc;
        }
        for (int m = 0; m < 5; m++)
            if ((rc = pz(slots[m], kz[m])) || (rc = px(slots[m], kx[m]))) return rc;
    }
    // force spectra S_c = ST_c(mu d_c psi) (:996-1027) and the Stokes velocity (:1030-1286)
    if (L.stokes_true_k && L.use_rd && L.use_rdz && L.use_multi && rd_len(L.g.nx) && rd_len(L.g.ny) &&
        rd_len(L.g.nz)) {
        // the order of adv_force_stokes_true_k: force spectra by true wavenumber, aligned
        // projection; the z passes that store or read one index up run over the pool, Sx's
        // x pass (one index up) per member
        auto pz_up = [&](int slot, bool store) {
            return on_pool_copy(L, [&](Ctx &pc) {
                pc.g.nx = L.g.nx * M;
#ifdef SMADFT_CHECK_BOUNDS
                pc.g.nelem = L.g.nelem * M;
#endif
                T *f = L.f<T>(slot);
                return store ? z_pass_upstore<T>(pc, f, f) : z_pass_upread<T>(pc, f, f);
            });
        };
        for (int i = 0; i < M; i++) {
            rc = on_lead_stream(L, *mm[i], [&](Ctx &c) {
                Spec<T> s = make_spec<T>(c);
                T *psi = c.f<T>(S_PSI), *sp2 = c.f<T>(S_SP2);
                const KindSet<3> ks{{K_DCT2, K_DST2, K_DCT2}};
                const auto lm = make_multi(LdForce<T>{psi, sp2, c.f<T>(S_GX), s.beta, s.gamma},
                                           LdForce<T>{psi, sp2, c.f<T>(S_GY), s.beta, s.gamma},
                                           LdForce<T>{psi, sp2, c.f<T>(S_GZ), s.beta, s.gamma});
                const StoreMultiUp<T, 3, 1> sm{{c.f<T>(S_SX), c.f<T>(S_SY), c.f<T>(S_SZ)}, 2u, (idx_t)c.g.nz, c.g.ny};
                using LM = std::remove_const_t<decltype(lm)>;
                using SM = StoreMultiUp<T, 3, 1>;
                switch (c.g.ny) {
                case 64: return launch_rd<T, 64, 1, LM, SM, 3, 1>(c, ks, lm, sm);
                case 128: return launch_rd<T, 128, 1, LM, SM, 3, 1>(c, ks, lm, sm);
                default: return launch_rd<T, 256, 1, LM, SM, 3, 1>(c, ks, lm, sm);
                }
            });
            if (rc) return rc;
        }
        if ((rc = pz(S_SX, K_DCT2)) || (rc = pz(S_SY, K_DCT2)) || (rc = pz_up(S_SZ, true))) return rc;
        for (int i = 0; i < M; i++) {
            rc = on_lead_stream(L, *mm[i], [&](Ctx &c) {
                T *Sx = c.f<T>(S_SX);
                return launch_axis<T, 0>(c, K_DST2, LoadArr<T>{Sx}, StoreUp<T, 0>{Sx, (idx_t)c.g.nyz, c.g.nx});
            });
            if (rc) return rc;
        }
        if ((rc = px(S_SY, K_DCT2)) || (rc = px(S_SZ, K_DCT2))) return rc;
        const int ky[3] = {K_DCT3, K_DST3, K_DCT3};
        for (int i = 0; i < M; i++) {
            rc = on_lead_stream(L, *mm[i], [&](Ctx &c) {
                Spec<T> s = make_spec<T>(c);
                T *Sx = c.f<T>(S_SX), *Sy = c.f<T>(S_SY), *Sz = c.f<T>(S_SZ);
                T *const out[3] = {c.f<T>(S_VX), c.f<T>(S_VY), c.f<T>(S_VZ)};
                return y_pass_multi<T, 3, 0>(c, ky, out, LdStokesK<T, 0>{s, Sx, Sy, Sz}, LdStokesK<T, 1>{s, Sx, Sy, Sz},
                                             LdStokesK<T, 2>{s, Sx, Sy, Sz});
            });
            if (rc) return rc;
        }
        if ((rc = pz(S_VX, K_DCT3)) || (rc = px(S_VX, K_DST3)) || (rc = pz(S_VY, K_DCT3)) ||
            (rc = px(S_VY, K_DCT3)) || (rc = pz_up(S_VZ, false)) || (rc = px(S_VZ, K_DCT3)))
            return rc;
    } else {
        {
            const int kx[3] = {K_DST2, K_DCT2, K_DCT2};
            const int ky[3] = {K_DCT2, K_DST2, K_DCT2};
            const int kz[3] = {K_DCT2, K_DCT2, K_DST2};
            const int slots[3] = {S_SX, S_SY, S_SZ};
            for (int i = 0; i < M; i++) {
                rc = on_lead_stream(L, *mm[i], [&](Ctx &c) {
                    Spec<T> s = make_spec<T>(c);
                    T *psi = c.f<T>(S_PSI), *sp2 = c.f<T>(S_SP2);
                    T *const out[3] = {c.f<T>(S_SX), c.f<T>(S_SY), c.f<T>(S_SZ)};
                    return y_pass_multi<T, 3, 1>(c, ky, out, LdForce<T>{psi, sp2, c.f<T>(S_GX), s.beta, s.gamma},
                                                 LdForce<T>{psi, sp2, c.f<T>(S_GY), s.beta, s.gamma},
                                                 LdForce<T>{psi, sp2, c.f<T>(S_GZ), s.beta, s.gamma});
                });
                if (rc) return rc;
            }
            for (int m = 0; m < 3; m++)
                if ((rc = pz(slots[m], kz[m])) || (rc = px(slots[m], kx[m]))) return rc;
        }
        // Stokes velocity (:1030-1286)
        {
            const int kx[3] = {K_DST3, K_DCT3, K_DCT3};
            const int ky[3] = {K_DCT3, K_DST3, K_DCT3};
            const int kz[3] = {K_DCT3, K_DCT3, K_DST3};
            const int slots[3] = {S_VX, S_VY, S_VZ};
            for (int i = 0; i < M; i++) {
                rc = on_lead_stream(L, *mm[i], [&](Ctx &c) {
                    Spec<T> s = make_spec<T>(c);
                    T *Sx = c.f<T>(S_SX), *Sy = c.f<T>(S_SY), *Sz = c.f<T>(S_SZ);
                    T *const out[3] = {c.f<T>(S_VX), c.f<T>(S_VY), c.f<T>(S_VZ)};
                    return y_pass_multi<T, 3, 0>(c, ky, out, LdStokes<T, 0, false>{s, Sx, Sy, Sz, nullptr},
                                                 LdStokes<T, 1, false>{s, Sx, Sy, Sz, nullptr},
                                                 LdStokes<T, 2, false>{s, Sx, Sy, Sz, nullptr});
                });
                if (rc) return rc;
            }
            for (int m = 0; m < 3; m++)
                if ((rc = pz(slots[m], kz[m])) || (rc = px(slots[m], kx[m]))) return rc;
        }
    }
    // N = beta psi^3 - gamma psi^5 - v.grad psi into the scratch field, CN/AB2 update (:1290-1365)
    for (int i = 0; i < M; i++) {
        rc = on_lead_stream(L, *mm[i], [&](Ctx &c) {
            Spec<T> s = make_spec<T>(c);
            return launch_axis<T, 1>(c, K_DCT2,
                                     LdAdvN<T>{c.f<T>(S_PSI), c.f<T>(S_VX), c.f<T>(S_VY), c.f<T>(S_VZ), c.f<T>(S_GX),
                                               c.f<T>(S_GY), c.f<T>(S_GZ), s.beta, s.gamma},
                                     StoreArr<T>{c.f<T>(S_TMP)});
        });
        if (rc) return rc;
    }
    if ((rc = pz(S_TMP, K_DCT2))) return rc;
    for (int i = 0; i < M; i++) {
        rc = on_lead_stream(L, *mm[i], [&](Ctx &c) {
            return launch_axis<T, 0>(c, K_DCT2, LoadArr<T>{c.f<T>(S_TMP)},
                                     StUpdCN<T>{make_spec<double>(c), c.f<double>(S_PSIH), c.f<T>(S_NP)});
        });
        if (rc) return rc;
    }
    return SMADFT_OK;
}

// each precision builds as its own object (SMADFT_INST_FLOAT / SMADFT_INST_DOUBLE); a plain
// compile without either instantiates both
#if !defined(SMADFT_INST_DOUBLE)
template int adv_fields<float>(Ctx &);
template int adv_step<float>(Ctx &);
template int adv_group_step<float>(Ctx *const *, int);
#endif
#if !defined(SMADFT_INST_FLOAT)
template int adv_fields<double>(Ctx &);
template int adv_step<double>(Ctx &);
template int adv_group_step<double>(Ctx *const *, int);
#endif

}  // namespace smadft
