// step_noadv.cu -- the diffusive loop body and the shared transform helpers.
#include "models.cuh"
#include "quasi.cuh"
#include "steps.h"

namespace smadft {

template <typename T>
int noadv_step(Ctx &c, bool keep_old)
{
    Spec<T> s = make_spec<T>(c);
    T *psi = c.f<T>(S_PSI);
    double *ph = c.f<double>(S_PSIH);   // spectral state (FP64)
    T *np = c.f<T>(S_NP);
    // N^n = REDFT10^3(beta psi^3 - gamma psi^5), fused CN/AB2 update of psihat (q^2-weighted
    // operator and N for conserved runs)
    int rc = c.p.conserved ? r2r3d<T>(c, K_DCT2, K_DCT2, K_DCT2, LdNonlin<T>{psi, s.beta, s.gamma},
                                      StUpdCN<T, 1>{make_spec<double>(c), ph, np})
                           : r2r3d<T>(c, K_DCT2, K_DCT2, K_DCT2, LdNonlin<T>{psi, s.beta, s.gamma},
                                      StUpdCN<T>{make_spec<double>(c), ph, np});
    if (rc) return rc;
    // psi^{n+1} = REDFT01^3 psihat (into the second buffer when the old psi is needed)
    T *dst = keep_old ? c.f<T>(S_PSI2) : psi;
    return r2r3d<T>(c, K_DCT3, K_DCT3, K_DCT3, LoadArr<T, double>{ph}, StoreArr<T>{dst});
}

// The diffusive loop body for M batch members of one grid with pooled fields (see
// adv_group_step): per member the nonlinearity's y pass and the CN/AB2 x pass (their
// functors carry the member's parameters), the plain passes once over the pool.
template <typename T>
int noadv_group_step(Ctx *const *mm, int M)
{
    Ctx &L = *mm[0];
    int rc;
    for (int i = 0; i < M; i++) {
        rc = on_lead_stream(L, *mm[i], [&](Ctx &c) {
            Spec<T> s = make_spec<T>(c);
            return launch_axis<T, 1>(c, K_DCT2, LdNonlin<T>{c.f<T>(S_PSI), s.beta, s.gamma}, StoreArr<T>{c.f<T>(S_TMP)});
        });
        if (rc) return rc;
    }
    if ((rc = pooled_pass<T, 2>(L, M, K_DCT2, L.f<T>(S_TMP), L.f<T>(S_TMP)))) return rc;
    for (int i = 0; i < M; i++) {
        rc = on_lead_stream(L, *mm[i], [&](Ctx &c) {
            return launch_axis<T, 0>(c, K_DCT2, LoadArr<T>{c.f<T>(S_TMP)},
                                     StUpdCN<T>{make_spec<double>(c), c.f<double>(S_PSIH), c.f<T>(S_NP)});
        });
        if (rc) return rc;
    }
    // psi^{n+1} = REDFT01^3 psihat, all members at once
    if ((rc = pooled_pass<T, 1, double>(L, M, K_DCT3, L.f<double>(S_PSIH), L.f<T>(S_TMP)))) return rc;
    if ((rc = pooled_pass<T, 2>(L, M, K_DCT3, L.f<T>(S_TMP), L.f<T>(S_TMP)))) return rc;
    return pooled_pass<T, 0>(L, M, K_DCT3, L.f<T>(S_TMP), L.f<T>(S_PSI));
}

template <typename T>
int refresh_psi(Ctx &c, T *dst)
{
    return r2r3d<T>(c, K_DCT3, K_DCT3, K_DCT3, LoadArr<T, double>{c.f<double>(S_PSIH)}, StoreArr<T>{dst});
}

template <typename T>
int pre_loop(Ctx &c)
{
    Spec<T> s = make_spec<T>(c);
    T *psi = c.f<T>(S_PSI);
    double *ph = c.f<double>(S_PSIH);
    T *np = c.f<T>(S_NP);
    int rc;
    if (c.p.model == SMADFT_MODEL_QUASI) return quasi_pre_loop<T>(c);
    if (c.p.model == SMADFT_MODEL_COMP) return comp_pre_loop<T>(c);
    // psihat = scale REDFT10^3 psi ; Nprev = REDFT10^3(beta psi^3 - gamma psi^5) (no advection)
    // no-adv/cosNoAdvTrackSing.cpp:618-635, adv/cosAdvTrackMult.cpp:760-777; weighted by q^2
    // for conserved noadv (no-adv/cosNoAdvConserv.cpp:688-701), unweighted for conserved adv
    // (adv/cosAdvConSingle.cpp:762-780)
    if ((rc = r2r3d<T>(c, K_DCT2, K_DCT2, K_DCT2, LoadArr<T>{psi}, StScale<T>{ph, c.scale}))) return rc;
    if (c.p.conserved && c.p.model == SMADFT_MODEL_NOADV)
        rc = r2r3d<T>(c, K_DCT2, K_DCT2, K_DCT2, LdNonlin<T>{psi, s.beta, s.gamma}, StQ2<T>{make_spec<double>(c), np});
    else
        rc = r2r3d<T>(c, K_DCT2, K_DCT2, K_DCT2, LdNonlin<T>{psi, s.beta, s.gamma}, StoreArr<T>{np});
    if (rc) return rc;
    return SMADFT_OK;
}

template <typename T>
int dfd_field(Ctx &c, T *dst)
{
    Spec<T> s = make_spec<T>(c);
    return r2r3d<T>(c, K_DCT3, K_DCT3, K_DCT3, LdDfd<T>{s, c.f<double>(S_PSIH)}, StoreArr<T>{dst});
}

template <typename T>
int psihat_from_psi(Ctx &c)
{
    return r2r3d<T>(c, K_DCT2, K_DCT2, K_DCT2, LoadArr<T>{c.f<T>(S_PSI)}, StScale<T>{c.f<double>(S_PSIH), c.scale});
}

template <typename T>
int plain_r2r3d(Ctx &c, const T *in, T *out, int kx, int ky, int kz)
{
    return r2r3d<T>(c, kx, ky, kz, LoadArr<T>{in}, StoreArr<T>{out});
}

template <typename T>
int plain_pass(Ctx &c, const T *in, T *out, int axis, int kind)
{
    return launch_pass<T>(c, axis, kind, LoadArr<T>{in}, StoreArr<T>{out});
}

#define SMADFT_INST(T)                                                      \
    template int noadv_step<T>(Ctx &, bool);                               \
    template int refresh_psi<T>(Ctx &, T *);                               \
    template int pre_loop<T>(Ctx &);                                       \
    template int dfd_field<T>(Ctx &, T *);                                 \
    template int psihat_from_psi<T>(Ctx &);                                \
    template int plain_r2r3d<T>(Ctx &, const T *, T *, int, int, int);     \
    template int plain_pass<T>(Ctx &, const T *, T *, int, int);          \
    template int noadv_group_step<T>(Ctx *const *, int);
// each precision builds as its own object (SMADFT_INST_FLOAT / SMADFT_INST_DOUBLE); a plain
// compile without either instantiates both
#if !defined(SMADFT_INST_DOUBLE)
SMADFT_INST(float)
#endif
#if !defined(SMADFT_INST_FLOAT)
SMADFT_INST(double)
#endif
#undef SMADFT_INST

}  // namespace smadft
