// ref_host_shim.cpp -- extern "C" probe into the reference's own host classes
// (TEST INFRASTRUCTURE, built only into oracle/_ref/libref_host.so by
// oracle/ref.mk).  It constructs the reference's InputVariables / Params /
// Params2 / Psi / Vext / Output exactly as its main.cu and plugins do and
// copies the results out, so tests can pin this project's host mirror
// (fgpe_b200/host) against the reference bit for bit.  No reference code is
// copied here; the reference sources are compiled where they lie.
#include "input_variables.hpp"
#include "output.hpp"
#include "params.hpp"
#include "params2.hpp"
#include "psi.hpp"
#include "vext.hpp"

#include <cstring>

namespace {
// Layout of the dump array shared with tests/refhost.py:
//  [0..2] NX  [3] DIM  [4] Npoints  [5..7] XMAX  [8..10] DX  [11] DV
//  [12..14] KXMAX  [15..17] DKX  [18] V  [19] dt  [20] epsilon_e  [21] time0
//  [22] niter  [23] itmod  [24] aho(1)  [25] omho(1)  [26..28] ax(1)
//  [29..31] omega(1)  [32] mass(1)  [33] npart(1)  [34] a / a11  [35] add / a22
//  [36] edd / a12  [37] aho2  [38] omho2  [39..41] ax2  [42..44] omega2
//  [45] mass2  [46] npart2
const int DUMP_N = 47;

void fill_base(const ParamsBase& p, double* o) {
    for (int i = 0; i < 3; ++i) o[i] = p.NX[i];
    o[3] = p.DIM;
    o[4] = p.Npoints;
    for (int i = 0; i < 3; ++i) {
        o[5 + i] = p.XMAX[i];
        o[8 + i] = p.DX[i];
        o[12 + i] = p.KXMAX[i];
        o[15 + i] = p.DKX[i];
    }
    o[11] = p.DV;
    o[18] = p.V;
    o[19] = p.dt;
    o[20] = p.epsilon_e;
    o[21] = p.time0;
    o[22] = p.niter;
    o[23] = p.itmod;
}
}  // namespace

extern "C" {

int ref_dump_len(void) { return DUMP_N; }

// Params (t2component false) or Params2 (true), main.cu:34-71.
int ref_params(const char* file, double* o) {
    std::memset(o, 0, sizeof(double) * DUMP_N);
    InputVariables reader{std::string(file)};
    if (!reader.getBool("t2component")) {
        Params p(reader);
        fill_base(p, o);
        o[24] = p.aho; o[25] = p.omho;
        for (int i = 0; i < 3; ++i) { o[26 + i] = p.ax[i]; o[29 + i] = p.omega[i]; }
        o[32] = p.mass; o[33] = p.npart; o[34] = p.a; o[35] = p.add; o[36] = p.edd;
        return 1;
    }
    Params2 p(reader);
    fill_base(p, o);
    o[24] = p.aho1; o[25] = p.omho1;
    for (int i = 0; i < 3; ++i) { o[26 + i] = p.ax1[i]; o[29 + i] = p.omega1[i]; }
    o[32] = p.mass1; o[33] = p.npart1; o[34] = p.a11; o[35] = p.a22; o[36] = p.a12;
    o[37] = p.aho2; o[38] = p.omho2;
    for (int i = 0; i < 3; ++i) { o[39 + i] = p.ax2[i]; o[42 + i] = p.omega2[i]; }
    o[45] = p.mass2; o[46] = p.npart2;
    return 2;
}

// Psi of the 1-component plugin, hamiltonians/BEC_oneComponent.cu:36-58
// (construction + optional vortex imprint), or component `type` (1, 2) of
// hamiltonians/BEC_twoComponent.cu:41-73.
int ref_init_psi(const char* file, int type, double* out) {
    InputVariables reader{std::string(file)};
    if (!reader.getBool("t2component")) {
        Params p(reader);
        Psi* ps = new Psi(p, std::string(""));
        if (p.getBool("tpi_vortex")) ps->imprintVortexTube(p, p.getDouble("api_prc"));
        std::memcpy(out, ps->getPsi(), sizeof(complex) * p.Npoints);
        delete ps;
        return 0;
    }
    Params2 p(reader);
    Psi* ps = new Psi(p, type);
    if (p.getBool("tpi_vortex")) ps->imprintVortexTube(p, p.getDouble("api_prc"));
    std::memcpy(out, ps->getPsi(), sizeof(complex) * p.Npoints);
    delete ps;
    return 0;
}

// The one-component Psi of ref_init_psi with one of the reference's lattice
// seeds applied (src/psi.cu:179-348); lattice numbering as gpeh_init_psi_lattice.
int ref_init_psi_lattice(const char* file, int lattice, double amp, double k, double offx, double offy,
                         double offz, int type, double* out) {
    InputVariables reader{std::string(file)};
    Params p(reader);
    Psi* ps = new Psi(p, std::string(""));
    if (p.getBool("tpi_vortex")) ps->imprintVortexTube(p, p.getDouble("api_prc"));
    switch (lattice) {
        case 1: ps->force1DLattice(p, amp, k, offx, type); break;
        case 2: ps->force2DTriangularLattice(p, amp, k, offx, offy, type); break;
        case 3: ps->force2DSquareLattice(p, amp, k, offx, offy, type); break;
        case 4: ps->force3DHEXLattice(p, amp, k, offx, offy, offz, type); break;
        case 5: ps->force3DFCCLattice(p, amp, k, offx, offy, offz, type); break;
        case 6: ps->force3DBCCLattice(p, amp, k, offx, offy, offz, type); break;
        case 7: ps->force3DSCLattice(p, amp, k, offx, offy, offz, type); break;
        default: delete ps; return -1;
    }
    std::memcpy(out, ps->getPsi(), sizeof(complex) * p.Npoints);
    delete ps;
    return 0;
}

// Vext of the plugins, hamiltonians/BEC_oneComponent.cu:63-83 and
// hamiltonians/BEC_twoComponent.cu:80-110.
int ref_init_vext(const char* file, int type, double* out) {
    InputVariables reader{std::string(file)};
    if (!reader.getBool("t2component")) {
        Params p(reader);
        Vext* v = new Vext(p, std::string(""));
        if (p.getBool("tvseed")) v->addProtocolPotential(p, 0);
        std::memcpy(out, v->getVext(), sizeof(complex) * p.Npoints);
        delete v;
        return 0;
    }
    Params2 p(reader);
    Vext* v = new Vext(p, type);
    if (p.getBool("tvseed")) v->addWeightedProtocolPotential(p, type);
    std::memcpy(out, v->getVext(), sizeof(complex) * p.Npoints);
    delete v;
    return 0;
}

// Output::WriteWtxt / WriteWtxt_2c followed by WriteVariable2WTXT lines
// (src/output.cu:26-191), written under the input file's outprefix.
int ref_write_info(const char* file, int ncycles, int nvars, const char** names,
                   const double* values, const char** units) {
    InputVariables reader{std::string(file)};
    if (!reader.getBool("t2component")) {
        Params p(reader);
        Output out(p.outpath);
        out.WriteWtxt(p, ncycles);
        for (int i = 0; i < nvars; ++i) out.WriteVariable2WTXT(names[i], values[i], units[i]);
        return 0;
    }
    Params2 p(reader);
    Output out(p.outpath);
    out.WriteWtxt_2c(p, ncycles);
    for (int i = 0; i < nvars; ++i) out.WriteVariable2WTXT(names[i], values[i], units[i]);
    return 0;
}

}  // extern "C"
