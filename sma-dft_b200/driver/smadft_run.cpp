// smadft_run -- reference-style host driver over the smadft C ABI.
//
// It keeps the reference's driver surface (parameter block, IC builders, output files) and
// calls the library once per loop body.  Output files follow the reference's names and
// text formats: L1.dat (no-adv/cosNoAdvTrackSing.cpp:789-795), surfPsi.dat, velSurf.dat,
// curvH.dat, curvK.dat, psiMid.dat (:1004-1030), vx/vy/vz.dat mid slices (adv/cosAdvTrackMult.cpp:1613-1731), mass.dat and
// energy.dat (quasi/quasi.cpp:2232-2248), info (quasi/quasi.cpp:820-843), and the per-rank
// text save psi0.dat (adv/cosAdvTrackMult.cpp:1546-1557) which `ic=file:` reads back.
//
// quasi also writes the divv.dat, p.dat, rho.dat and energyMid.dat mid slices of its save
// iteration (quasi/quasi.cpp:91-126,2466-2487).
// comp (compressible/compressible.cpp) also writes rhoMid.dat and amp.dat mid slices
// (:2885-2892) and rho0.dat at the end (:2786-2799), and tracks rho > rho_s - 0.15 (:2734).
//
// usage: smadft_run noadv|adv|quasi|comp [nu e0d radius load] [key=value ...]
//   keys: n nx ny nz nw dt eps alpha beta gamma nu kp rho0 divv steps l1every saveevery
//         precision(fp64|fp32) conserved(0|1) ic(interface|bump|focal|conics|file:<path>) A
//         radius seed noise out track_axis track_mode track_hi track_lo checkpoint resume
//         zeta rhoup (comp)
// conserved=1 runs the reference's conserved variants (no-adv/cosNoAdvConserv.cpp,
// adv/cosAdvConSingle.cpp); their save iteration writes surfPsi.dat but no velSurf/curvH/curvK
// values (the library has no conserved surface diagnostics).
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <map>
#include <string>
#include <vector>

#include "smadft.h"

namespace {

struct Opt {
    std::map<std::string, std::string> kv;
    std::string get(const std::string &k, const std::string &d) const
    {
        auto it = kv.find(k);
        return it == kv.end() ? d : it->second;
    }
    double num(const std::string &k, double d) const
    {
        auto it = kv.find(k);
        return it == kv.end() ? d : std::atof(it->second.c_str());
    }
};

int die(const char *what, int rc, smadft_ctx *ctx)
{
    std::fprintf(stderr, "smadft_run: %s failed: %s (%d)%s%s\n", what, smadft_error_string(rc), rc,
                 ctx ? " -- " : "", ctx ? smadft_last_error(ctx) : "");
    return 1;
}

void append_slice(const std::string &path, const std::vector<double> &f, int nx, int ny, int nz)
{
    std::ofstream o(path, std::ios_base::app);
    const int j = ny / 2;
    for (int i = 0; i < nx; i++)
        for (int k = 0; k < nz; k++) o << f[((size_t)i * ny + j) * nz + k] << "\n";
}

}  // namespace

int main(int argc, char **argv)
{
    if (argc < 2) {
        std::fprintf(stderr, "usage: %s noadv|adv|quasi|comp [nu e0d radius load] [key=value ...]\n", argv[0]);
        return 2;
    }
    std::string model = argv[1];
    int m = model == "noadv" ? SMADFT_MODEL_NOADV : model == "adv" ? SMADFT_MODEL_ADV
          : model == "quasi" ? SMADFT_MODEL_QUASI : model == "comp" ? SMADFT_MODEL_COMP : -1;
    if (m < 0) { std::fprintf(stderr, "unknown model %s\n", argv[1]); return 2; }
    Opt o;
    std::vector<std::string> pos;
    for (int a = 2; a < argc; a++) {
        std::string s = argv[a];
        size_t eq = s.find('=');
        if (eq == std::string::npos) pos.push_back(s);
        else o.kv[s.substr(0, eq)] = s.substr(eq + 1);
    }
    smadft_params p;
    smadft_params_init(&p, m);
    // reference argv: nu, eps = -0.01 arg (adv) or -0.001 arg (quasi), radius, load
    // (adv/cosAdvTrackMult.cpp:127,160-177; quasi/quasi.cpp:173,221-240)
    if (pos.size() >= 1) p.nu = std::atof(pos[0].c_str());
    if (pos.size() >= 2) p.eps = (m >= SMADFT_MODEL_QUASI ? -0.001 : -0.01) * std::atof(pos[1].c_str());
    if (pos.size() >= 3) o.kv.emplace("radius", pos[2]);
    if (pos.size() >= 4 && std::atoi(pos[3].c_str()) == 1) {
        o.kv.emplace("ic", "file:psi0.dat");
        p.loaded = (m == SMADFT_MODEL_QUASI);
    }
    int n = (int)o.num("n", 64);
    p.nx = (int)o.num("nx", n); p.ny = (int)o.num("ny", n); p.nz = (int)o.num("nz", n);
    p.nw = o.num("nw", p.nw); p.dt = o.num("dt", p.dt); p.eps = o.num("eps", p.eps);
    p.alpha = o.num("alpha", p.alpha); p.beta = o.num("beta", p.beta); p.gamma = o.num("gamma", p.gamma);
    p.nu = o.num("nu", p.nu); p.kp = o.num("kp", p.kp); p.rho0 = o.num("rho0", p.rho0);
    p.divv_switch = (int)o.num("divv", p.divv_switch);
    p.zeta = o.num("zeta", p.zeta);
    p.rho_up = (int)o.num("rhoup", p.rho_up);
    p.precision = o.get("precision", "fp64") == "fp32" ? SMADFT_FP32 : SMADFT_FP64;
    p.conserved = (int)o.num("conserved", 0);
    const long steps = (long)o.num("steps", 1000);
    const bool dens = m == SMADFT_MODEL_QUASI || m == SMADFT_MODEL_COMP;   // models with a density
    const int l1every = (int)o.num("l1every", dens ? 50 : 100);
    const int saveevery = (int)o.num("saveevery", 10);
    const std::string out = o.get("out", ".") + "/";
    const int taxis = (int)o.num("track_axis", 2);
    const int tmode = (int)o.num("track_mode", dens ? SMADFT_TRACK_LEVEL : SMADFT_TRACK_FLAT);
    // quasi: rho > rho_0 + 0.2 (quasi/quasi.cpp:2264-2280); comp: rho > rho_s - 0.15 with
    // rho_s = 1 (compressible/compressible.cpp:2734)
    const double thi = o.num("track_hi", m == SMADFT_MODEL_QUASI ? p.rho0 + 0.2 : m == SMADFT_MODEL_COMP ? 0.85 : 0.7);
    const double tlo = o.num("track_lo", 0.0);
    int rc = smadft_params_check(&p);
    if (rc) return die("parameter check", rc, nullptr);

    const size_t N = (size_t)p.nx * p.ny * p.nz;
    std::vector<double> psi(N);
    std::string ic = o.get("ic", "interface");
    const double A = o.num("A", 1.328);
    const unsigned long long seed = (unsigned long long)o.num("seed", 20240601);
    const double noise = o.num("noise", 1e-3);
    if (ic == "interface") rc = smadft_ic_interface(&p, A, 0.0, noise, seed, psi.data());
    else if (ic == "bump") rc = smadft_ic_interface(&p, A, 2.0 * 2.0 * M_PI / p.q0, noise, seed, psi.data());
    else if (ic == "focal") rc = smadft_ic_focal_conic(&p, A, o.num("radius", p.nx / 2.0), psi.data());
    else if (ic == "conics") rc = smadft_ic_conics(&p, A, 4, 3.0, 6.0, noise, seed, psi.data());
    else if (ic.rfind("file:", 0) == 0) {
        std::ifstream f(ic.substr(5));
        if (!f.is_open()) { std::fprintf(stderr, "cannot open %s\n", ic.c_str() + 5); return 1; }
        for (size_t q = 0; q < N; q++) f >> psi[q];
        rc = f.fail() ? SMADFT_ERR_IO : SMADFT_OK;
    } else {
        std::fprintf(stderr, "unknown ic %s\n", ic.c_str());
        return 2;
    }
    if (rc) return die("initial condition", rc, nullptr);

    smadft_ctx *ctx = nullptr;
    if ((rc = smadft_create(&p, &ctx))) return die("smadft_create", rc, nullptr);
    if ((rc = smadft_set_psi(ctx, psi.data(), N))) return die("smadft_set_psi", rc, ctx);
    if (o.kv.count("resume") && (rc = smadft_load_checkpoint(ctx, o.get("resume", "").c_str())))
        return die("resume", rc, ctx);

    {   // files are created empty, as the reference does at start-up
        for (const char *f : {"L1.dat", "psiMid.dat", "surfPsi.dat"}) std::ofstream(out + f).close();
        if (!dens)
            for (const char *f : {"velSurf.dat", "curvH.dat", "curvK.dat"}) std::ofstream(out + f).close();
        if (m != SMADFT_MODEL_NOADV) for (const char *f : {"vx.dat", "vy.dat", "vz.dat"}) std::ofstream(out + f).close();
        if (dens) for (const char *f : {"mass.dat", "energy.dat"}) std::ofstream(out + f).close();
        if (m == SMADFT_MODEL_COMP) for (const char *f : {"rhoMid.dat", "amp.dat"}) std::ofstream(out + f).close();
        if (m == SMADFT_MODEL_QUASI)   // quasi/quasi.cpp:872,926-936
            for (const char *f : {"divv.dat", "rho.dat", "p.dat", "energyMid.dat"}) std::ofstream(out + f).close();
        std::ofstream info(out + "info");
        info << "Nx: " << p.nx << "\nNy: " << p.ny << "\nNz: " << p.nz << "\nPoints per wavelength (nw): "
             << p.nw << "\nq0 (z direction): " << p.q0 << "\nepsilon: " << p.eps << "\nbeta: " << p.beta
             << "\ngamma: " << p.gamma << "\nViscosity (nu): " << p.nu << "\ndt: " << p.dt
             << "\nprecision: " << (p.precision == SMADFT_FP32 ? "fp32" : "fp64")
             << "\nconserved: " << p.conserved << "\n";
    }
    long done = 0;
    int countSave = 0;
    std::vector<double> field(N);
    const int na = taxis == 0 ? p.ny : p.nx, nb = taxis == 2 ? p.ny : p.nz;
    std::vector<int> sidx((size_t)na * nb);
    std::vector<double> spos((size_t)na * nb), vel((size_t)na * nb), cH((size_t)na * nb), cK((size_t)na * nb);
    // the reference's own save iteration (z-scanning flat tracker, noadv / adv) also writes the
    // normal velocity and curvatures of that step (no-adv/cosNoAdvTrackSing.cpp:808-1021,
    // adv/cosAdvTrackMult.cpp:1311-1585)
    const bool with_surface = !dens && !p.conserved && taxis == 2 && tmode == SMADFT_TRACK_FLAT;
    while (done < steps) {
        long chunk = std::min<long>(l1every - 1, steps - done - 1);
        if (chunk > 0 && (rc = smadft_step(ctx, (int)chunk))) return die("smadft_step", rc, ctx);
        done += chunk;
        smadft_diag d;
        const bool surf_iter = with_surface && countSave + 1 == saveevery;
        rc = surf_iter ? smadft_step_surface(ctx, sidx.data(), vel.data(), cH.data(), cK.data(), &d)
                       : smadft_step_diag(ctx, &d);
        done++;
        if (rc == SMADFT_ERR_NONFINITE) {
            std::fprintf(stderr, "smadft_run: psi became non-finite at step %ld\n", done);
            return 3;
        }
        if (rc) return die("smadft_step_diag", rc, ctx);
        std::ofstream(out + "L1.dat", std::ios_base::app) << std::setprecision(17) << d.l1 << "\n";
        if (dens) {
            std::ofstream(out + "mass.dat", std::ios_base::app) << std::setprecision(17) << d.mass << "\n";
            std::ofstream(out + "energy.dat", std::ios_base::app) << std::setprecision(17) << d.energy << "\n";
        }
        if (++countSave == saveevery) {
            countSave = 0;
            int fld = (dens && tmode == SMADFT_TRACK_LEVEL) ? SMADFT_FIELD_RHO : SMADFT_FIELD_PSI;
            if (!surf_iter && (rc = smadft_track(ctx, fld, taxis, tmode, thi, tlo, sidx.data(), spos.data())))
                return die("smadft_track", rc, ctx);
            {
                std::ofstream s(out + "surfPsi.dat", std::ios_base::app);
                for (size_t q = 0; q < sidx.size(); q++) s << sidx[q] << "\n";
            }
            if (surf_iter) {
                const std::vector<double> *v[3] = {&vel, &cH, &cK};
                const char *names[3] = {"velSurf.dat", "curvH.dat", "curvK.dat"};
                for (int c = 0; c < 3; c++) {
                    std::ofstream s(out + names[c], std::ios_base::app);
                    s << std::setprecision(17);
                    for (double x : *v[c]) s << x << "\n";
                }
            }
            if ((rc = smadft_get_psi(ctx, field.data(), N))) return die("smadft_get_psi", rc, ctx);
            append_slice(out + "psiMid.dat", field, p.nx, p.ny, p.nz);
            if (m == SMADFT_MODEL_COMP) {
                int ids[2] = {SMADFT_FIELD_RHO, SMADFT_FIELD_AMP};
                const char *names[2] = {"rhoMid.dat", "amp.dat"};
                for (int c = 0; c < 2; c++) {
                    if ((rc = smadft_get_field(ctx, ids[c], field.data(), N))) return die("smadft_get_field", rc, ctx);
                    append_slice(out + names[c], field, p.nx, p.ny, p.nz);
                }
            }
            if (m == SMADFT_MODEL_QUASI) {
                // saveMid of div v (real space), pressure, density and energy density at
                // j = Ny/2 (quasi/quasi.cpp:91-126,2466-2487)
                int ids[4] = {SMADFT_FIELD_DIVV_REAL, SMADFT_FIELD_P, SMADFT_FIELD_RHO, SMADFT_FIELD_ENERGY};
                const char *names[4] = {"divv.dat", "p.dat", "rho.dat", "energyMid.dat"};
                for (int c = 0; c < 4; c++) {
                    if ((rc = smadft_get_field(ctx, ids[c], field.data(), N))) return die("smadft_get_field", rc, ctx);
                    append_slice(out + names[c], field, p.nx, p.ny, p.nz);
                }
            }
            if (m != SMADFT_MODEL_NOADV) {
                int ids[3] = {SMADFT_FIELD_VX, SMADFT_FIELD_VY, SMADFT_FIELD_VZ};
                const char *names[3] = {"vx.dat", "vy.dat", "vz.dat"};
                for (int c = 0; c < 3; c++) {
                    if ((rc = smadft_get_field(ctx, ids[c], field.data(), N))) return die("smadft_get_field", rc, ctx);
                    append_slice(out + names[c], field, p.nx, p.ny, p.nz);
                }
            }
            if (o.kv.count("checkpoint") && (rc = smadft_save_checkpoint(ctx, o.get("checkpoint", "").c_str())))
                return die("checkpoint", rc, ctx);
            std::cout << "The loop " << done << " finished" << std::endl;
        }
    }
    if ((rc = smadft_get_psi(ctx, psi.data(), N))) return die("smadft_get_psi", rc, ctx);
    {
        std::ofstream s(out + "psi0.dat");
        s << std::setprecision(17);
        for (size_t q = 0; q < N; q++) s << psi[q] << "\n";
    }
    if (m == SMADFT_MODEL_COMP) {   // the density save beside psi (compressible/compressible.cpp:2786-2799)
        if ((rc = smadft_get_field(ctx, SMADFT_FIELD_RHO, psi.data(), N))) return die("smadft_get_field", rc, ctx);
        std::ofstream s(out + "rho0.dat");
        s << std::setprecision(17);
        for (size_t q = 0; q < N; q++) s << psi[q] << "\n";
    }
    smadft_destroy(ctx);
    return 0;
}
