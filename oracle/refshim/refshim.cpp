/*
 * refshim.cpp -- implementation of the single-rank FFTW-MPI / MPI stand-in declared in
 * fftw3-mpi.h (test infrastructure: it only links the reference's own sources into
 * oracle/_ref).  Transforms run through the oracle's FP64 r2r (oracle/r2r.c).
 */
#include "fftw3-mpi.h"

#include <cstdio>
#include <cstdlib>
#include <string>

extern "C" {
#include "r2r.h"
}

namespace MPI {
const Datatype DOUBLE = {8};
const Op SUM = {0};
Intracomm COMM_WORLD;
} // namespace MPI

struct refshim_plan_s {
    ptrdiff_t n0, n1, n2;
    double *in, *out;
    int k[3];
};

static int map_kind(fftw_r2r_kind k)
{
    switch (k) {
    case FFTW_REDFT10: return ORC_REDFT10;
    case FFTW_REDFT01: return ORC_REDFT01;
    case FFTW_RODFT10: return ORC_RODFT10;
    case FFTW_RODFT01: return ORC_RODFT01;
    default:
        std::fprintf(stderr, "refshim: r2r kind %d is not provided\n", (int)k);
        std::abort();
    }
}

void fftw_mpi_init(void) {}

ptrdiff_t fftw_mpi_local_size_3d(ptrdiff_t n0, ptrdiff_t n1, ptrdiff_t n2, MPI_Comm,
                                 ptrdiff_t *local_n0, ptrdiff_t *local_0_start)
{
    *local_n0 = n0;
    *local_0_start = 0;
    return n0 * n1 * n2;
}

fftw_plan fftw_mpi_plan_r2r_3d(ptrdiff_t n0, ptrdiff_t n1, ptrdiff_t n2, double *in, double *out,
                               MPI_Comm, fftw_r2r_kind k0, fftw_r2r_kind k1, fftw_r2r_kind k2,
                               unsigned)
{
    refshim_plan_s *p = new refshim_plan_s;
    p->n0 = n0; p->n1 = n1; p->n2 = n2;
    p->in = in; p->out = out;
    p->k[0] = map_kind(k0); p->k[1] = map_kind(k1); p->k[2] = map_kind(k2);
    return p;
}

void fftw_execute(const fftw_plan p)
{
    orc_r2r_3d(p->in, p->out, (int)p->n0, (int)p->n1, (int)p->n2, p->k[0], p->k[1], p->k[2]);
}

void fftw_destroy_plan(fftw_plan p) { delete p; }
void fftw_cleanup(void) {}

double refshim_param(const char *key, double def)
{
    std::string name = std::string("REFSHIM_") + key;
    const char *s = std::getenv(name.c_str());
    return s ? std::atof(s) : def;
}

long refshim_steps(void)
{
    const char *s = std::getenv("REFSHIM_STEPS");
    return s ? std::atol(s) : 0;
}

const char *refshim_dir(void)
{
    const char *s = std::getenv("REFSHIM_DIR");
    return s ? s : ".";
}

void refshim_load_ic(double *psi, ptrdiff_t n)
{
    const char *path = std::getenv("REFSHIM_IC");
    if (!path || !*path) return;
    FILE *f = std::fopen(path, "rb");
    if (!f) { std::fprintf(stderr, "refshim: cannot open IC %s\n", path); std::abort(); }
    size_t got = std::fread(psi, sizeof(double), (size_t)n, f);
    std::fclose(f);
    if (got != (size_t)n) { std::fprintf(stderr, "refshim: IC %s is short\n", path); std::abort(); }
}

void refshim_dump(const char *name, const double *v, ptrdiff_t n)
{
    std::string path = std::string(refshim_dir()) + "/" + name + ".bin";
    FILE *f = std::fopen(path.c_str(), "wb");
    if (!f) { std::fprintf(stderr, "refshim: cannot write %s\n", path.c_str()); std::abort(); }
    std::fwrite(v, sizeof(double), (size_t)n, f);
    std::fclose(f);
}
