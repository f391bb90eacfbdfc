#!/usr/bin/env bash
# build_ref.sh -- compile the reference's own time-step sources into oracle/_ref/ (test
# infrastructure: the binaries pin the oracle and give the CPU baseline).
#
# The sources are read where they lie (SMADFT_REFERENCE, default: a "reference" directory
# beside this repository) and are
# never copied into the repository: each one is streamed through sed into g++ on stdin.
# FFTW and MPI are not installed, so the build links the single-rank shim in refshim/.
# The sed edits only turn hard-coded constants into run-time parameters and add hooks:
#   * N, Nw, dt, eps, nu, kp, rho_0, divvSwitch      -> refshim_param("<KEY>", ref default)
#   * while (L1 > limL1)                              -> a fixed count, REFSHIM_STEPS
#   * the IC block is kept; refshim_load_ic() may overwrite psi afterwards (REFSHIM_IC)
#   * output directories                              -> REFSHIM_DIR
#   * psiMid's hard-coded j = 256 (noadv Sing)        -> Ny/2 (in range for small grids)
#   * L1/mass/energy/velSurf/curvH/curvK text output  -> 17 significant digits
#   * before MPI::Finalize(), binary dumps of the final fields
# Usage: oracle/build_ref.sh   (writes oracle/_ref/{noadv,bump,adv,quasi,noadvc,advc,comp}_ref)
set -euo pipefail
HERE="$(cd "$(dirname "$0")" && pwd)"
REF="${SMADFT_REFERENCE:-$HERE/../../reference}"
OUT="$HERE/_ref"
CXX="${SMADFT_CXX:-g++}"
CC="${SMADFT_CC:-gcc}"
if [ ! -d "$REF" ]; then
    echo "build_ref.sh: reference sources not found at $REF" >&2
    exit 2
fi
mkdir -p "$OUT"
$CC -O2 -fopenmp -fPIC -c "$HERE/r2r.c" -I"$HERE" -o "$OUT/r2r.o"
$CXX -O2 -fopenmp -fPIC -c "$HERE/refshim/refshim.cpp" -I"$HERE/refshim" -I"$HERE" -o "$OUT/refshim.o"

P='refshim_param'
COMMON=(
  -e "s/const ptrdiff_t Nx = [0-9]*, Ny = [0-9]*, Nz = [0-9]*;/const ptrdiff_t Nx = (ptrdiff_t)$P(\"NX\", 64), Ny = (ptrdiff_t)$P(\"NY\", 64), Nz = (ptrdiff_t)$P(\"NZ\", 64);/"
  -e "s/const int    Nw = \([0-9]*\);/const int    Nw = (int)$P(\"NW\", \1);/"
  -e "s/const double dt = \([0-9.]*\);/const double dt = $P(\"DT\", \1);/"
  -e "s/const double gamma =  \([0-9.]*\);/const double gamma = $P(\"GAMMA\", \1);/"
  -e "s/const double beta  =  \([0-9.]*\);/const double beta = $P(\"BETA\", \1);/"
  -e "s/const double alpha =  \([0-9.]*\);/const double alpha = $P(\"ALPHA\", \1);/"
  -e "s/while (L1 > limL1)/for (long refshim_s = 0; refshim_s < refshim_steps(); refshim_s++)/"
  -e "s/L1_output << L1 << /L1_output << std::setprecision(17) << L1 << /"
  -e "s/velS_output << velSurf\[index\] << /velS_output << std::setprecision(17) << velSurf[index] << /"
  -e "s/curvH_output << curvH\[index\] << /curvH_output << std::setprecision(17) << curvH[index] << /"
  -e "s/curvK_output << curvK\[index\] << /curvK_output << std::setprecision(17) << curvK[index] << /"
)

build() { # name source extra-sed-args... ; dump statement is passed in DUMP
    local name="$1" src="$2"; shift 2
    sed "${COMMON[@]}" "$@" -e "s|MPI::Finalize();|$DUMP MPI::Finalize();|" "$REF/$src" |
        $CXX -std=c++11 -O2 -fopenmp -x c++ -I"$HERE/refshim" - -x none \
            "$OUT/refshim.o" "$OUT/r2r.o" -lm -o "$OUT/$name"
    echo "built $OUT/$name from $src"
}

# no-adv/cosNoAdvTrackSing.cpp
DUMP='refshim_dump("psi", psi_local.data(), alloc_local); refshim_dump("nq", Nq_local.data(), alloc_local);'
build noadv_ref no-adv/cosNoAdvTrackSing.cpp \
  -e "s/const double ep    = \([-0-9.]*\);/const double ep = $P(\"EPS\", \1);/" \
  -e "s|^\(\s*\)// Generate psiq for substrate gradient penalty|\1refshim_load_ic(psi_local.data(), alloc_local);|" \
  -e "s/^\(\s*\)j = 256;/\1j = Ny\/2;/" \
  -e "s|std::ofstream L1_output(\"L1.dat\");|std::ofstream L1_output(std::string(refshim_dir()) + \"/L1.dat\");|" \
  -e "s|L1_output.open(\"L1.dat\",|L1_output.open(std::string(refshim_dir()) + \"/L1.dat\",|"

# no-adv/cosNoAdvTrackBump.cpp (bump tracker); load switched off, IC through the hook
DUMP='refshim_dump("psi", psi_local.data(), alloc_local);'
build bump_ref no-adv/cosNoAdvTrackBump.cpp \
  -e "s/const double ep    = \([-0-9.]*\);/const double ep = $P(\"EPS\", \1);/" \
  -e "s/int load = 1;/int load = 0;/" \
  -e "s|std::string strLoad = \"box4/save/\";|std::string strLoad = std::string(refshim_dir()) + \"/\";|" \
  -e "s|std::string strBox = \"box4/saveBump/\";|std::string strBox = std::string(refshim_dir()) + \"/\";|" \
  -e "s|^\(\s*\)// Generate psiq for substrate gradient penalty|\1refshim_load_ic(psi_local.data(), alloc_local);|"

# adv/cosAdvTrackMult.cpp; argv = nu e0d radius load (the directory names use them)
DUMP='refshim_dump("psi", psi_local.data(), alloc_local); refshim_dump("vx", velx_local.data(), alloc_local); refshim_dump("vy", vely_local.data(), alloc_local); refshim_dump("vz", velz_local.data(), alloc_local); refshim_dump("gx", psiGradx_local.data(), alloc_local); refshim_dump("gy", psiGrady_local.data(), alloc_local); refshim_dump("gz", psiGradz_local.data(), alloc_local); refshim_dump("nq", Nq_local.data(), alloc_local);'
build adv_ref adv/cosAdvTrackMult.cpp \
  -e "s/const double ep = -0.01\*ep_arg;/const double ep = $P(\"EPS\", -0.01*ep_arg);/" \
  -e "s/double nu = atof(argv\[1\]);/double nu = $P(\"NU\", atof(argv[1]));/" \
  -e "s|std::string strLoad = \"[^\"]*\";|std::string strLoad = std::string(refshim_dir()) + \"/r\";|" \
  -e "s|std::string strBox = \"[^\"]*\";|std::string strBox = std::string(refshim_dir()) + \"/r\";|" \
  -e "s|^\(\s*\)// Generate psiq for substrate gradient penalty|\1refshim_load_ic(psi_local.data(), alloc_local);|"

# quasi/quasi.cpp; argv = nu e0d radius load
DUMP='refshim_dump("psi", psi_local.data(), alloc_local); refshim_dump("rho", rho_local.data(), alloc_local); refshim_dump("p", p_local.data(), alloc_local); refshim_dump("vx", velx_local.data(), alloc_local); refshim_dump("vy", vely_local.data(), alloc_local); refshim_dump("vz", velz_local.data(), alloc_local); refshim_dump("mu", mu_local.data(), alloc_local); refshim_dump("energy", energy_local.data(), alloc_local); refshim_dump("psiq", psiq_local.data(), alloc_local);'
build quasi_ref quasi/quasi.cpp \
  -e "s/const double ep = -0.001\*ep_arg;/const double ep = $P(\"EPS\", -0.001*ep_arg);/" \
  -e "s/double nu = atof(argv\[1\]);/double nu = $P(\"NU\", atof(argv[1]));/" \
  -e "s/double rho_0 = \([0-9.]*\);/double rho_0 = $P(\"RHO0\", \1);/" \
  -e "s/double kp = \([0-9.]*\);/double kp = $P(\"KP\", \1);/" \
  -e "s/const int divvSwitch = \([0-9]*\);/const int divvSwitch = (int)$P(\"DIVV\", \1);/" \
  -e "s|std::string strLoad = \"[^\"]*\";|std::string strLoad = std::string(refshim_dir()) + \"/r\";|" \
  -e "s|std::string strBox = \"[^\"]*\";|std::string strBox = std::string(refshim_dir()) + \"/r\";|" \
  -e "s|mass_output << rho_sum << |mass_output << std::setprecision(17) << rho_sum << |" \
  -e "s|energy_output << energy << |energy_output << std::setprecision(17) << energy << |" \
  -e "s|^\(\s*\)/\*\* Create output files \*\*/|\1refshim_load_ic(psi_local.data(), alloc_local);|"

# no-adv/cosNoAdvConserv.cpp (conserved dynamics); argv = e0d radius N load
DUMP='refshim_dump("psi", psi_local.data(), alloc_local); refshim_dump("nq", Nq_local.data(), alloc_local);'
build noadvc_ref no-adv/cosNoAdvConserv.cpp \
  -e "s/const ptrdiff_t Nx = atof(argv\[3\]), Ny = atof(argv\[3\]), Nz = atof(argv\[3\]);/const ptrdiff_t Nx = (ptrdiff_t)$P(\"NX\", 64), Ny = (ptrdiff_t)$P(\"NY\", 64), Nz = (ptrdiff_t)$P(\"NZ\", 64);/" \
  -e "s/const double ep = -0.01\*ep_arg;/const double ep = $P(\"EPS\", -0.01*ep_arg);/" \
  -e "s|std::string strLoad = \"[^\"]*\";|std::string strLoad = std::string(refshim_dir()) + \"/r\";|" \
  -e "s|std::string strBox = \"[^\"]*\";|std::string strBox = std::string(refshim_dir()) + \"/r\";|" \
  -e "s|^\(\s*\)// Generate psiq for substrate gradient penalty|\1refshim_load_ic(psi_local.data(), alloc_local);|"

# adv/cosAdvConSingle.cpp (conserved dynamics); argv = nu e0d radius N load
DUMP='refshim_dump("psi", psi_local.data(), alloc_local); refshim_dump("vx", velx_local.data(), alloc_local); refshim_dump("vy", vely_local.data(), alloc_local); refshim_dump("vz", velz_local.data(), alloc_local); refshim_dump("gx", psiGradx_local.data(), alloc_local); refshim_dump("gy", psiGrady_local.data(), alloc_local); refshim_dump("gz", psiGradz_local.data(), alloc_local); refshim_dump("nq", Nq_local.data(), alloc_local);'
build advc_ref adv/cosAdvConSingle.cpp \
  -e "s/const ptrdiff_t Nx = atof(argv\[4\]), Ny = atof(argv\[4\]), Nz = atof(argv\[4\]);/const ptrdiff_t Nx = (ptrdiff_t)$P(\"NX\", 64), Ny = (ptrdiff_t)$P(\"NY\", 64), Nz = (ptrdiff_t)$P(\"NZ\", 64);/" \
  -e "s/const double ep = -0.01\*ep_arg;/const double ep = $P(\"EPS\", -0.01*ep_arg);/" \
  -e "s/double nu = atof(argv\[1\]);/double nu = $P(\"NU\", atof(argv[1]));/" \
  -e "s|std::string strLoad = \"[^\"]*\";|std::string strLoad = std::string(refshim_dir()) + \"/r\";|" \
  -e "s|std::string strBox = \"[^\"]*\";|std::string strBox = std::string(refshim_dir()) + \"/r\";|" \
  -e "s|^\(\s*\)// Generate psiq for substrate gradient penalty|\1refshim_load_ic(psi_local.data(), alloc_local);|"

# compressible/compressible.cpp (independent density, amplitude field); argv = nu e0d radius load
DUMP='refshim_dump("psi", psi_local.data(), alloc_local); refshim_dump("rho", rho_local.data(), alloc_local); refshim_dump("psiq", psiq_local.data(), alloc_local); refshim_dump("amp", amp_local.data(), alloc_local); refshim_dump("divv", divv_local.data(), alloc_local); refshim_dump("mu", mu_local.data(), alloc_local); refshim_dump("vsolx", vsolx_local.data(), alloc_local); refshim_dump("vsoly", vsoly_local.data(), alloc_local); refshim_dump("vsolz", vsolz_local.data(), alloc_local); refshim_dump("virrx", virrx_local.data(), alloc_local); refshim_dump("virry", virry_local.data(), alloc_local); refshim_dump("virrz", virrz_local.data(), alloc_local); refshim_dump("nl", Nl_local.data(), alloc_local); refshim_dump("frho", f_rho_local.data(), alloc_local);'
build comp_ref compressible/compressible.cpp \
  -e "s/const double ep = -0.001\*ep_arg;/const double ep = $P(\"EPS\", -0.001*ep_arg);/" \
  -e "s/double nu = atof(argv\[1\]);/double nu = $P(\"NU\", atof(argv[1]));/" \
  -e "s/double rho_0 = \([0-9.]*\);/double rho_0 = $P(\"RHO0\", \1);/" \
  -e "s/double zeta = \([0-9.]*\);/double zeta = $P(\"ZETA\", \1);/" \
  -e "s/const int divvSwitch = \([0-9]*\);/const int divvSwitch = (int)$P(\"DIVV\", \1);/" \
  -e "s/const int rhoUP = \([0-9]*\);/const int rhoUP = (int)$P(\"RHO_UP\", \1);/" \
  -e "s|std::string strLoad = \"[^\"]*\";|std::string strLoad = std::string(refshim_dir()) + \"/\";|" \
  -e "s|std::string strSave = \"[^\"]*\";|std::string strSave = std::string(refshim_dir()) + \"/\";|" \
  -e "s|std::string strBox = \"[^\"]*\";|std::string strBox = std::string(refshim_dir()) + \"/\";|" \
  -e "s|mass_output << rho_sum << |mass_output << std::setprecision(17) << rho_sum << |" \
  -e "s|energy_output << energy << |energy_output << std::setprecision(17) << energy << |" \
  -e "s|^\(\s*\)/\*\* Create output files \*\*/|\1refshim_load_ic(psi_local.data(), alloc_local);|"
