// host_capi.cpp -- C entry points of the host mirror (include/gpe_host.h).
#include <cstring>

#include "../../include/gpe_host.h"
#include "gpe_host.hpp"

namespace {
thread_local std::string g_host_err;
const int DUMP_N = 47;

void fill_base(const gpe::ParamsBase& p, double* o) {
    for (int i = 0; i < 3; ++i) {
        o[i] = p.NX[i];
        o[5 + i] = p.XMAX[i];
        o[8 + i] = p.DX[i];
        o[12 + i] = p.KXMAX[i];
        o[15 + i] = p.DKX[i];
    }
    o[3] = p.DIM;
    o[4] = p.Npoints;
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

int gpeh_dump_len(void) { return DUMP_N; }

const char* gpeh_last_error(void) { return g_host_err.c_str(); }

int gpeh_params(const char* file, double* o) {
    try {
        std::memset(o, 0, sizeof(double) * DUMP_N);
        gpe::InputVariables iv{std::string(file)};
        if (!iv.getBool("t2component")) {
            gpe::Params p(iv);
            fill_base(p, o);
            o[24] = p.aho;
            o[25] = p.omho;
            for (int i = 0; i < 3; ++i) {
                o[26 + i] = p.ax[i];
                o[29 + i] = p.omega[i];
            }
            o[32] = p.mass;
            o[33] = p.npart;
            o[34] = p.a;
            o[35] = p.add;
            o[36] = p.edd;
            return 1;
        }
        gpe::Params2 p(iv);
        fill_base(p, o);
        o[24] = p.aho1;
        o[25] = p.omho1;
        for (int i = 0; i < 3; ++i) {
            o[26 + i] = p.ax1[i];
            o[29 + i] = p.omega1[i];
            o[39 + i] = p.ax2[i];
            o[42 + i] = p.omega2[i];
        }
        o[32] = p.mass1;
        o[33] = p.npart1;
        o[34] = p.a11;
        o[35] = p.a22;
        o[36] = p.a12;
        o[37] = p.aho2;
        o[38] = p.omho2;
        o[45] = p.mass2;
        o[46] = p.npart2;
        return 2;
    } catch (const std::exception& e) {
        g_host_err = e.what();
        return -1;
    }
}

int gpeh_init_psi(const char* file, int type, double* out) {
    try {
        gpe::InputVariables iv{std::string(file)};
        if (!iv.getBool("t2component")) {
            gpe::Params p(iv);
            gpe::Psi ps(p, std::string(""));
            if (p.getBool("tpi_vortex")) ps.imprintVortexTube(p, p.getDouble("api_prc"));
            std::memcpy(out, ps.psi.data(), sizeof(gpe::complex) * p.Npoints);
            return 0;
        }
        gpe::Params2 p(iv);
        gpe::Psi ps(p, type);
        if (p.getBool("tpi_vortex")) ps.imprintVortexTube(p, p.getDouble("api_prc"));
        std::memcpy(out, ps.psi.data(), sizeof(gpe::complex) * p.Npoints);
        return 0;
    } catch (const std::exception& e) {
        g_host_err = e.what();
        return -1;
    }
}

int gpeh_init_psi_lattice(const char* file, int lattice, double amp, double k, double offx, double offy,
                          double offz, int type, double* out) {
    try {
        gpe::InputVariables iv{std::string(file)};
        gpe::Params p(iv);
        gpe::Psi ps(p, std::string(""));
        if (p.getBool("tpi_vortex")) ps.imprintVortexTube(p, p.getDouble("api_prc"));
        switch (lattice) {
            case 1: ps.force1DLattice(p, amp, k, offx, type); break;
            case 2: ps.force2DTriangularLattice(p, amp, k, offx, offy, type); break;
            case 3: ps.force2DSquareLattice(p, amp, k, offx, offy, type); break;
            case 4: ps.force3DHEXLattice(p, amp, k, offx, offy, offz, type); break;
            case 5: ps.force3DFCCLattice(p, amp, k, offx, offy, offz, type); break;
            case 6: ps.force3DBCCLattice(p, amp, k, offx, offy, offz, type); break;
            case 7: ps.force3DSCLattice(p, amp, k, offx, offy, offz, type); break;
            default: throw gpe::HostError("unknown lattice " + std::to_string(lattice));
        }
        std::memcpy(out, ps.psi.data(), sizeof(gpe::complex) * p.Npoints);
        return 0;
    } catch (const std::exception& e) {
        g_host_err = e.what();
        return -1;
    }
}

int gpeh_init_vext(const char* file, int type, double* out) {
    try {
        gpe::InputVariables iv{std::string(file)};
        if (!iv.getBool("t2component")) {
            gpe::Params p(iv);
            gpe::Vext v(p, std::string(""));
            if (p.getBool("tvseed")) v.addProtocolPotential(p, 0);
            std::memcpy(out, v.vext.data(), sizeof(gpe::complex) * p.Npoints);
            return 0;
        }
        gpe::Params2 p(iv);
        gpe::Vext v(p, type);
        if (p.getBool("tvseed")) v.addWeightedProtocolPotential(p, type);
        std::memcpy(out, v.vext.data(), sizeof(gpe::complex) * p.Npoints);
        return 0;
    } catch (const std::exception& e) {
        g_host_err = e.what();
        return -1;
    }
}

int gpeh_write_info(const char* file, int ncycles, int nvars, const char** names, const double* values,
                    const char** units) {
    try {
        gpe::InputVariables iv{std::string(file)};
        if (!iv.getBool("t2component")) {
            gpe::Params p(iv);
            gpe::Output out(p.outpath);
            out.WriteWtxt(p, ncycles);
            for (int i = 0; i < nvars; ++i) out.WriteVariable2WTXT(names[i], values[i], units[i]);
            return 0;
        }
        gpe::Params2 p(iv);
        gpe::Output out(p.outpath);
        out.WriteWtxt_2c(p, ncycles);
        for (int i = 0; i < nvars; ++i) out.WriteVariable2WTXT(names[i], values[i], units[i]);
        return 0;
    } catch (const std::exception& e) {
        g_host_err = e.what();
        return -1;
    }
}

int gpeh_run(const char* file) { return gpe::run_input_file(std::string(file)); }

}  // extern "C"
