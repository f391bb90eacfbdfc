/*
 * fftw3-mpi.h -- single-rank stand-in for FFTW-MPI and the MPI C++ bindings, used only
 * to compile the reference's own sources into oracle/_ref (test infrastructure).
 *
 * The reference includes <fftw3-mpi.h> and relies on it for <mpi.h> as well.  Neither
 * FFTW nor MPI is installed here, so this header declares exactly the subset the three
 * canonical sources call (see the API list below) with one-rank semantics:
 *   - Get_rank() == 0, Get_size() == 1;
 *   - Gather/Scatter copy sendbuf -> recvbuf; Reduce copies; Bcast/Barrier do nothing;
 *   - Send/Recv address ranks that do not exist on one rank and are no-ops that leave the
 *     buffers untouched (the reference's halo planes then stay zero-filled);
 *   - fftw_mpi_local_size_3d gives the whole box to rank 0;
 *   - fftw_execute runs the 3-D r2r transform of the plan with the oracle's FP64 r2r
 *     (oracle/r2r.c, checked against scipy's DCT/DST, which follow FFTW's definitions).
 * It also declares the hooks that oracle/build_ref.sh splices into the sources
 * (fixed step count, IC injection, binary dumps).
 */
#ifndef SMADFT_REFSHIM_FFTW3_MPI_H
#define SMADFT_REFSHIM_FFTW3_MPI_H

#include <cstddef>
#include <cstring>

typedef int MPI_Comm;

namespace MPI {

struct Datatype {
    int size;
};
struct Op {
    int id;
};
extern const Datatype DOUBLE;
extern const Op SUM;

struct Intracomm {
    int Get_rank() const { return 0; }
    int Get_size() const { return 1; }
    void Barrier() const {}
    void Bcast(void *, int, const Datatype &, int) const {}
    void Send(const void *, int, const Datatype &, int, int) const {}
    void Recv(void *, int, const Datatype &, int, int) const {}
    void Gather(const void *s, int sc, const Datatype &t, void *r, int, const Datatype &, int) const
    {
        if (s != r) std::memmove(r, s, (size_t)sc * (size_t)t.size);
    }
    void Scatter(const void *s, int sc, const Datatype &t, void *r, int, const Datatype &, int) const
    {
        if (s != r) std::memmove(r, s, (size_t)sc * (size_t)t.size);
    }
    void Reduce(const void *s, void *r, int c, const Datatype &t, const Op &, int) const
    {
        if (s != r) std::memmove(r, s, (size_t)c * (size_t)t.size);
    }
    operator MPI_Comm() const { return 0; }
};
extern Intracomm COMM_WORLD;

inline void Init() {}
inline void Finalize() {}

} // namespace MPI

typedef enum {
    FFTW_REDFT00, FFTW_REDFT01, FFTW_REDFT10, FFTW_REDFT11,
    FFTW_RODFT00, FFTW_RODFT01, FFTW_RODFT10, FFTW_RODFT11
} fftw_r2r_kind;

#define FFTW_MEASURE 0u
#define FFTW_ESTIMATE (1u << 6)

typedef struct refshim_plan_s *fftw_plan;

void fftw_mpi_init(void);
ptrdiff_t fftw_mpi_local_size_3d(ptrdiff_t n0, ptrdiff_t n1, ptrdiff_t n2, MPI_Comm comm,
                                 ptrdiff_t *local_n0, ptrdiff_t *local_0_start);
fftw_plan fftw_mpi_plan_r2r_3d(ptrdiff_t n0, ptrdiff_t n1, ptrdiff_t n2, double *in, double *out,
                               MPI_Comm comm, fftw_r2r_kind k0, fftw_r2r_kind k1, fftw_r2r_kind k2,
                               unsigned flags);
void fftw_execute(const fftw_plan p);
void fftw_destroy_plan(fftw_plan p);
void fftw_cleanup(void);

/* hooks spliced in by oracle/build_ref.sh */
double refshim_param(const char *key, double def);        /* REFSHIM_<key>, else def */
long refshim_steps(void);                                 /* REFSHIM_STEPS, default 0 */
const char *refshim_dir(void);                            /* REFSHIM_DIR, default "." */
void refshim_load_ic(double *psi, ptrdiff_t n);           /* REFSHIM_IC binary file, if set */
void refshim_dump(const char *name, const double *v, ptrdiff_t n); /* REFSHIM_DIR/<name>.bin */

#endif
