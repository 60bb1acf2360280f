// psi_vext_output.cpp -- initial states, potentials and output files (host
// mirror of src/psi.cu, src/vext.cu, src/output.cu; same arithmetic order and
// file formats, so a run writes the same bytes the reference writes).
#include <algorithm>
#include <cmath>
#include <iostream>

#include "gpe_host.hpp"

namespace gpe {

double gridX(const ParamsBase& p, int i) {
    int ix = i % p.NX[0];
    return -p.XMAX[0] + (ix)*p.DX[0] + 0.5 * p.DX[0];
}
double gridY(const ParamsBase& p, int i) {
    int iy = (i / p.NX[0]) % p.NX[1];
    return -p.XMAX[1] + (iy)*p.DX[1] + 0.5 * p.DX[1];
}
double gridZ(const ParamsBase& p, int i) {
    int iz = i / (p.NX[0] * p.NX[1]);
    return -p.XMAX[2] + (iz)*p.DX[2] + 0.5 * p.DX[2];
}

namespace {
bool any_zero(const double* om) {
    return std::any_of(om, om + 3, [](double x) { return std::abs(x) < 1E-6; });
}
}  // namespace

// ---- Psi ------------------------------------------------------------------------
Psi::Psi(const Params& p, const std::string&) : generator(p.getInt("rndseed")) {
    psi.assign(p.Npoints, complex(0, 0));
    if (p.getBool("read_psi")) {
        readPsi(p.inpath, p.Npoints);
    } else {
        if (any_zero(p.omega) && std::abs(p.omega[0]) < 1E-6) initTube(p, 0);
        else initHarmonic(p, 0);
        normalize(p);
    }
}

Psi::Psi(const ParamsBase& p, int type) : generator(p.getInt("rndseed") + type) {
    psi.assign(p.Npoints, complex(0, 0));
    if (p.getBool("read_psi")) {
        readPsi(p.inpath + std::to_string(type), p.Npoints);
    } else {
        const double* om = p._omega(type == 1 ? 1 : 2);
        if (any_zero(om) && std::abs(om[0]) < 1E-6) initTube(p, type);
        else initHarmonic(p, type);
        normalize(p, type);
    }
}

// The reference builds complex(rrnd*U(), crnd*U()) in one expression
// (src/psi.cu:93,112); with the GNU toolchain that builds it the imaginary
// argument's draw is evaluated first.  The draws are made explicit here in
// that order, which the host-mirror tests pin against the reference's build.
complex Psi::noise(double rrnd, double crnd) {
    const double ui = distribution(generator);
    const double ur = distribution(generator);
    return complex(rrnd * ur, crnd * ui);
}

void Psi::initTube(const ParamsBase& p, int type) {
    const double rrnd = p.getDouble("rand_pct");
    const double crnd = p.getDouble("crand_pct");
    const double* ax = p._ax(type == 1 ? 1 : (type == 2 ? 2 : 1));
    for (int i = 0; i < p.Npoints; ++i) {
        double y = gridY(p, i) / ax[1];
        double z = gridZ(p, i) / ax[2];
        complex n = noise(rrnd, crnd);
        psi[i] = (complex(1, 0) + n) * complex(std::exp(-0.5 * 0.1 * ((y * y) + (z * z))), 0);
    }
}

void Psi::initHarmonic(const ParamsBase& p, int type) {
    const double rrnd = p.getDouble("rand_pct");
    const double crnd = p.getDouble("crand_pct");
    const double* ax = p._ax(type == 1 ? 1 : (type == 2 ? 2 : 1));
    for (int i = 0; i < p.Npoints; ++i) {
        double x = gridX(p, i) / ax[0];
        double y = gridY(p, i) / ax[1];
        double z = gridZ(p, i) / ax[2];
        complex n = noise(rrnd, crnd);
        psi[i] = (complex(1, 0) + n) * complex(std::exp(-0.5 * 0.1 * ((y * y) + (z * z) + (x * x))), 0);
    }
}

// src/psi.cu:351-374
void Psi::normalize(const ParamsBase& p, int type) {
    double norm = 0;
    const double npart = (type == 1 || type == -1 || type == 0) ? p._npart(1) : p._npart(2);
    for (int i = 0; i < p.Npoints; ++i) norm += std::pow(std::abs(psi[i]), 2);
    norm = std::pow(npart / (norm * p.DX[0] * p.DX[1] * p.DX[2]), 0.5);
    for (int i = 0; i < p.Npoints; ++i) psi[i] = psi[i] * norm;
}

// src/psi.cu:155-164
void Psi::imprintVortexTube(const ParamsBase& p, double Ncirc) {
    const double xLen = 2 * p.XMAX[0];
    for (int i = 0; i < p.Npoints; ++i) {
        double x = gridX(p, i);
        psi[i] = complex(std::cos(Ncirc * 2 * pi / xLen * x), std::sin(Ncirc * 2 * pi / xLen * x)) * psi[i];
    }
}

// ---- lattice seeds, src/psi.cu:179-348 ---------------------------------------------
// shape(i) is the seed amplitude at point i; its cosine sums are grouped and
// ordered as the reference groups them, so the result is the same to the bit.
template <class Shape>
void Psi::add_lattice(const ParamsBase& p, int type, Shape shape) {
    const double npart = (type == 1) ? p._npart(1) : p._npart(2);
    const double avg = std::pow(npart / (p.DX[0] * p.DX[1] * p.DX[2]), 0.5);
    for (int i = 0; i < p.Npoints; ++i) psi[i] = shape(i) * avg + psi[i];
    normalize(p, 1);
}

void Psi::force1DLattice(const ParamsBase& p, double amp, double k, double off, int type) {
    add_lattice(p, type, [&](int i) {
        const double x = gridX(p, i) - off;
        return amp * (1 - std::cos(k * x)) / 2.;  // 0 .. amp
    });
}

void Psi::force2DTriangularLattice(const ParamsBase& p, double amp, double k, double offx, double offy, int type) {
    const double h = std::sqrt(3.0) / 2;  // sin 60 deg
    add_lattice(p, type, [&](int i) {
        const double x = gridX(p, i) - offx, y = gridY(p, i) - offy;
        return amp * (std::cos(k * x) + std::cos(k * (-0.5 * x + h * y)) + std::cos(k * (-0.5 * x - h * y))) / 3;
    });
}

void Psi::force2DSquareLattice(const ParamsBase& p, double amp, double k, double offx, double offy, int type) {
    add_lattice(p, type, [&](int i) {
        const double x = gridX(p, i) - offx, y = gridY(p, i) - offy;
        return amp * (std::cos(k * y) + std::cos(k * x)) / 2;
    });
}

void Psi::force3DHEXLattice(const ParamsBase& p, double amp, double k, double offx, double offy, double offz,
                            int type) {
    const double r3 = std::sqrt(3.);
    add_lattice(p, type, [&](int i) {
        const double x = gridX(p, i) - offx, y = gridY(p, i) - offy, z = gridZ(p, i) - offz;
        const double u = (-x + r3 * y) / 2., w = (-x - r3 * y) / 2.;  // the in-plane directions at +-120 deg
        return amp * (std::cos(k * u) + std::cos(k * x) + std::cos(k * z) + std::cos(k * w)) / 4.0;
    });
}

void Psi::force3DFCCLattice(const ParamsBase& p, double amp, double k, double offx, double offy, double offz,
                            int type) {
    const double r3 = std::sqrt(3.);
    add_lattice(p, type, [&](int i) {
        const double x = gridX(p, i) - offx, y = gridY(p, i) - offy, z = gridZ(p, i) - offz;
        // the nine projections of the reference, in its order
        const double q[9] = {(x + y - z) / r3, (y + z - x) / r3, (z + x - y) / r3,
                             (x - y - z) / r3, (y - z - x) / r3, (z - x - y) / r3,
                             (x + y + z) / r3, (y + z + x) / r3, (z + x + y) / r3};
        double s = std::cos(k * q[0]);
        for (int j = 1; j < 9; ++j) s = s + std::cos(k * q[j]);
        return amp * s / 9.0;
    });
}

void Psi::force3DBCCLattice(const ParamsBase& p, double amp, double k, double offx, double offy, double offz,
                            int type) {
    const double r2 = std::sqrt(2.0);
    add_lattice(p, type, [&](int i) {
        const double x = gridX(p, i) - offx, y = gridY(p, i) - offy, z = gridZ(p, i) - offz;
        const double q[6] = {(x + y) / r2, (z + y) / r2, (z + x) / r2, (x - y) / r2, (z - y) / r2, (z - x) / r2};
        double s = std::cos(k * q[0]);
        for (int j = 1; j < 6; ++j) s = s + std::cos(k * q[j]);
        return amp * s / 6;
    });
}

void Psi::force3DSCLattice(const ParamsBase& p, double amp, double k, double offx, double offy, double offz,
                           int type) {
    add_lattice(p, type, [&](int i) {
        const double x = gridX(p, i) - offx, y = gridY(p, i) - offy, z = gridZ(p, i) - offz;
        return amp * (std::cos(k * z) + std::cos(k * y) + std::cos(k * x)) / 3;
    });
}

// src/psi.cu:378-395 (a missing or short file is an error here, not a read
// from NULL).
void Psi::readPsi(const std::string& prefix, int length) {
    const std::string fn = prefix + "psi_final.wdat";
    FILE* f = std::fopen(fn.c_str(), "rb");
    if (!f) throw HostError("Could not open " + fn);
    size_t n = std::fread(psi.data(), sizeof(complex), length, f);
    std::fclose(f);
    if ((int)n != length)
        throw HostError("Only " + std::to_string(n) + " elements were read from " + fn + " instead of " +
                        std::to_string(length));
}

// ---- Vext --------------------------------------------------------------------------
Vext::Vext(const Params& p, const std::string&) {
    vext.assign(p.Npoints, complex(0, 0));
    if (p.getBool("read_vext")) {
        readVext(p.vpath, p.Npoints);
    } else if (any_zero(p.omega) && std::abs(p.omega[0]) < 1E-6) {
        initTube(p, 0);
    } else {
        initHarmonic(p, 0);
    }
}

Vext::Vext(const Params2& p, int type) {
    vext.assign(p.Npoints, complex(0, 0));
    if (p.getBool("read_vext")) {
        readVext(p.vpath + std::to_string(type), p.Npoints);
    } else {
        const double* om = p._omega(type == 1 ? 1 : 2);
        if (any_zero(om) && std::abs(om[0]) < 1E-6) initTube(p, type);
        else initHarmonic(p, type);
    }
}

// src/vext.cu:60-85
void Vext::initTube(const ParamsBase& p, int type) {
    const double* ax = p._ax(type == 2 ? 2 : 1);
    for (int i = 0; i < p.Npoints; ++i) {
        double y = gridY(p, i) / ax[1];
        double z = gridZ(p, i) / ax[2];
        vext[i] = 0.5 * (std::pow(y, 2) / std::pow(ax[1], 2) + std::pow(z, 2) / std::pow(ax[2], 2));
    }
}

void Vext::initHarmonic(const ParamsBase& p, int type) {
    const double* ax = p._ax(type == 2 ? 2 : 1);
    for (int i = 0; i < p.Npoints; ++i) {
        double x = gridX(p, i) / ax[0];
        double y = gridY(p, i) / ax[1];
        double z = gridZ(p, i) / ax[2];
        vext[i] = 0.5 * (std::pow(x, 2) / std::pow(ax[0], 2) + std::pow(y, 2) / std::pow(ax[1], 2) +
                         std::pow(z, 2) / std::pow(ax[2], 2));
    }
}

// src/vext.cu:201-218
void Vext::readVext(const std::string& prefix, int length) {
    const std::string fn = prefix + "vext.wdat";
    FILE* f = std::fopen(fn.c_str(), "rb");
    if (!f) throw HostError("Could not open the Vext file " + fn);
    size_t n = std::fread(vext.data(), sizeof(complex), length, f);
    std::fclose(f);
    if ((int)n != length)
        throw HostError("Only " + std::to_string(n) + " elements were read from " + fn + " instead of " +
                        std::to_string(length));
}

// src/vext.cu:152-165
void Vext::addProtocolPotential(const ParamsBase& p, int, int sign) {
    const double L = 2 * p.XMAX[0];
    const double n = p.getDouble("nseed");
    const double A = p.getDouble("aseed") * sign;
    for (int i = 0; i < p.Npoints; ++i) vext[i] += A * std::cos(n * 2 * pi / L * gridX(p, i));
}

// src/vext.cu:122-149
void Vext::addWeightedProtocolPotential(const Params2& p, int type) {
    const double n1 = p.npart1 / p.V;
    const double n2 = p.npart2 / p.V;
    const double c0 = p.getDouble("c0") / (p.aho1 * 1E-3);
    double A = 0;
    if (std::abs(c0) < 1E-6) {
        A = p.getDouble("aseed");
    } else {
        const double num = 4 * pi * (p.a11 - p.a12) - c0 * c0 / (n1 * p.omho1 * p.omho1);
        const double den = 4 * pi * (p.a22 - p.a12) - c0 * c0 / (n2 * p.omho1 * p.omho1);
        const double xi = -1 * num / den;
        if (xi > 0) A = (type == 1) ? 2 * p.getDouble("aseed") * xi / (1 + xi) : 2 * p.getDouble("aseed") / (1 + xi);
        else A = (type == 1) ? 2 * p.getDouble("aseed") * xi / (1 - xi) : 2 * p.getDouble("aseed") / (1 - xi);
    }
    const double L = 2 * p.XMAX[0];
    const double n = p.getDouble("nseed");
    for (int i = 0; i < p.Npoints; ++i) vext[i] += A * std::cos(n * 2 * pi / L * gridX(p, i));
}

// ---- Output (src/output.cu) ------------------------------------------------------------
namespace {
FILE* open_or_throw(const std::string& fn, const char* mode) {
    FILE* f = std::fopen(fn.c_str(), mode);
    if (!f) throw HostError("Could not open " + fn);
    return f;
}
}  // namespace

// src/output.cu:26-90.  The reference writes ly and lz with NX[0]
// (src/output.cu:42-44); that stays the default, so downstream readers see
// the same file.  The optional input key `wtxt_ref_lengths false` writes
// ly = NX[1] DX[1] aho and lz = NX[2] DX[2] aho instead.
void Output::WriteWtxt(const Params& p, int ncycle) {
    const bool ref_lengths =
        p.getIV().getVariable("wtxt_ref_lengths") == "None" || p.getBool("wtxt_ref_lengths");
    const int ny_l = ref_lengths ? p.NX[0] : p.NX[1];
    const int nz_l = ref_lengths ? p.NX[0] : p.NX[2];
    FILE* file = open_or_throw(prefix + "info.wtxt", "w");
    fprintf(file, "cycles                   %d\n\n", ncycle);
    fprintf(file, "dim                      %d\n", p.DIM);
    fprintf(file, "nx                       %d\n", p.NX[0]);
    fprintf(file, "ny                       %d\n", p.NX[1]);
    fprintf(file, "nz                       %d\n", p.NX[2]);
    fprintf(file, "dx                       %lf\n", p.DX[0]);
    fprintf(file, "dy                       %lf\n", p.DX[1]);
    fprintf(file, "dz                       %lf\n", p.DX[2]);
    fprintf(file, "lx                       %lf\n", p.NX[0] * p.DX[0] * p.aho);
    fprintf(file, "ly                       %lf\n", ny_l * p.DX[1] * p.aho);
    fprintf(file, "lz                       %lf\n", nz_l * p.DX[2] * p.aho);
    fprintf(file, "datadim                  %d\n", 3);
    fprintf(file, "prefix                   %s\n", p.outpath.c_str());
    fprintf(file, "t0                       %lf\n", p.time0);
    fprintf(file, "dt                       %lf\n\n", p.dt);
    fprintf(file, "%-15s %-15s %-15s %-15s %-15s\n", "# tag", "name", "value", "unit", "format");
    fprintf(file, "%-15s %-15s %-15s %-15s %-15s\n", "var", "psi", "complex", "none", "wdat");
    fprintf(file, "%-15s %-15s %-15s %-15s %-15s\n", "var", "vext", "complex", "none", "wdat");
    fprintf(file, "%-15s %-15s %-15s %-15s %-15s\n\n", "", "", "", "", "");
    fprintf(file, "%-15s %-15s %-15s %-15s\n", "# tag", "name", "value", "unit");
    fprintf(file, "%-15s %-15s %-15.1f %-15s\n", "const", "hbar       ", hbar, "u*(um)^2/s");
    fprintf(file, "%-15s %-15s %-15.1f %-15s\n", "const", "kB         ", kB, "[hbar]/nK");
    fprintf(file, "%-15s %-15s %-15.2f %-15s\n", "const", "npart      ", p.npart, "none");
    fprintf(file, "%-15s %-15s %-15.6f %-15s\n", "const", "mass       ", p.mass, "u");
    fprintf(file, "%-15s %-15s %-15.6E %-15s\n", "const", "abohr      ", abohr, "mu_m");
    fprintf(file, "%-15s %-15s %-15.6f %-15s\n", "const", "a          ", p.a / abohr * p.aho, "a0");
    if (p.getIV().getVariable("add") != "None") {
        fprintf(file, "%-15s %-15s %-15.6f %-15s\n", "const", "add        ", p.add / abohr * p.aho, "a0");
        fprintf(file, "%-15s %-15s %-15.6f %-15s\n", "const", "dipole_x   ", p.getDouble("dipole_x"), "1");
        fprintf(file, "%-15s %-15s %-15.6f %-15s\n", "const", "dipole_y   ", p.getDouble("dipole_y"), "1");
        fprintf(file, "%-15s %-15s %-15.6f %-15s\n", "const", "dipole_z   ", p.getDouble("dipole_z"), "1");
    }
    fprintf(file, "%-15s %-15s %-15.6f %-15s\n", "const", "omx        ", p.omega[0] / (2 * pi), "2pi");
    fprintf(file, "%-15s %-15s %-15.6f %-15s\n", "const", "omy        ", p.omega[1] / (2 * pi), "2pi");
    fprintf(file, "%-15s %-15s %-15.6f %-15s\n", "const", "omz        ", p.omega[2] / (2 * pi), "2pi");
    fprintf(file, "%-15s %-15s %-15.6f %-15s\n", "const", "aho        ", p.aho, "?");
    fprintf(file, "%-15s %-15s %-15.6f %-15s\n", "const", "ax         ", p.ax[0], "code");
    fprintf(file, "%-15s %-15s %-15.6f %-15s\n", "const", "ay         ", p.ax[1], "code");
    fprintf(file, "%-15s %-15s %-15.6f %-15s\n", "const", "az         ", p.ax[2], "code");
    fprintf(file, "%-15s %-15s %-15.6f %-15s\n", "const", "omho       ", p.omho, "?");
    fprintf(file, "%-15s %-15s %-15.1f %-15s\n", "const", "Eho        ", p.omho * hbar, "Energy_scale");
    fprintf(file, "%-15s %-15s %-15d %-15s\n", "const", "itmod      ", p.itmod, ".");
    fclose(file);
}

// src/output.cu:94-173
void Output::WriteWtxt_2c(const Params2& p, int ncycle) {
    FILE* file = open_or_throw(prefix + "info.wtxt", "w");
    fprintf(file, "cycles                   %d\n\n", ncycle);
    fprintf(file, "dim                      %d\n", p.DIM);
    fprintf(file, "nx                       %d\n", p.NX[0]);
    fprintf(file, "ny                       %d\n", p.NX[1]);
    fprintf(file, "nz                       %d\n", p.NX[2]);
    fprintf(file, "dx                       %lf\n", p.DX[0]);
    fprintf(file, "dy                       %lf\n", p.DX[1]);
    fprintf(file, "dz                       %lf\n", p.DX[2]);
    fprintf(file, "lx                       %lf\n", p.NX[0] * p.DX[0] * p.aho1);
    fprintf(file, "ly                       %lf\n", p.NX[1] * p.DX[1] * p.aho1);
    fprintf(file, "lz                       %lf\n", p.NX[2] * p.DX[2] * p.aho1);
    fprintf(file, "datadim                  %d\n", 3);
    fprintf(file, "prefix                   %s\n", p.outpath.c_str());
    fprintf(file, "t0                       %lf\n", p.time0);
    fprintf(file, "dt                       %lf\n\n", p.dt);
    fprintf(file, "%-15s %-15s %-15s %-15s %-15s\n", "# tag", "name", "value", "unit", "format");
    fprintf(file, "%-15s %-15s %-15s %-15s %-15s\n", "var", "1psi", "complex", "none", "wdat");
    fprintf(file, "%-15s %-15s %-15s %-15s %-15s\n", "var", "2psi", "complex", "none", "wdat");
    fprintf(file, "%-15s %-15s %-15s %-15s %-15s\n", "var", "1vext", "complex", "none", "wdat");
    fprintf(file, "%-15s %-15s %-15s %-15s %-15s\n", "var", "2vext", "complex", "none", "wdat");
    fprintf(file, "%-15s %-15s %-15s %-15s %-15s\n\n", "", "", "", "", "");
    fprintf(file, "%-15s %-15s %-15s %-15s\n", "# tag", "name", "value", "unit");
    fprintf(file, "%-15s %-15s %-15.1f %-15s\n", "const", "hbar       ", hbar, "u*(um)^2/s");
    fprintf(file, "%-15s %-15s %-15.1f %-15s\n", "const", "kB         ", kB, "[hbar]/nK");
    fprintf(file, "%-15s %-15s %-15.6E %-15s\n", "const", "abohr      ", abohr, "mu_m");
    fprintf(file, "%-15s %-15s %-15.1f %-15s\n", "const", "npart1      ", p.npart1, "none");
    fprintf(file, "%-15s %-15s %-15.6f %-15s\n", "const", "mass1       ", p.mass1, "u");
    fprintf(file, "%-15s %-15s %-15.6f %-15s\n", "const", "a11         ", p.a11 / abohr * p.aho1, "a0");
    fprintf(file, "%-15s %-15s %-15.1f %-15s\n", "const", "npart2      ", p.npart2, "none");
    fprintf(file, "%-15s %-15s %-15.6f %-15s\n", "const", "mass2       ", p.mass2, "u");
    fprintf(file, "%-15s %-15s %-15.6f %-15s\n", "const", "a22         ", p.a22 / abohr * p.aho1, "a0");
    fprintf(file, "%-15s %-15s %-15.6f %-15s\n", "const", "a12         ", p.a12 / abohr * p.aho1, "a0");
    fprintf(file, "%-15s %-15s %-15.2f %-15s\n", "const", "omx1        ", p.omega1[0] / (2 * pi), "2pi");
    fprintf(file, "%-15s %-15s %-15.2f %-15s\n", "const", "omy1        ", p.omega1[1] / (2 * pi), "2pi");
    fprintf(file, "%-15s %-15s %-15.2f %-15s\n", "const", "omz1        ", p.omega1[2] / (2 * pi), "2pi");
    fprintf(file, "%-15s %-15s %-15.2f %-15s\n", "const", "omx2        ", p.omega2[0] / (2 * pi), "2pi");
    fprintf(file, "%-15s %-15s %-15.2f %-15s\n", "const", "omy2        ", p.omega2[1] / (2 * pi), "2pi");
    fprintf(file, "%-15s %-15s %-15.2f %-15s\n", "const", "omz2        ", p.omega2[2] / (2 * pi), "2pi");
    fprintf(file, "%-15s %-15s %-15.6f %-15s\n", "const", "aho1        ", p.aho1, "?");
    fprintf(file, "%-15s %-15s %-15.6f %-15s\n", "const", "ax1         ", p.ax1[0], "code");
    fprintf(file, "%-15s %-15s %-15.6f %-15s\n", "const", "ay1         ", p.ax1[1], "code");
    fprintf(file, "%-15s %-15s %-15.6f %-15s\n", "const", "az1         ", p.ax1[2], "code");
    fprintf(file, "%-15s %-15s %-15.6f %-15s\n", "const", "omho1       ", p.omho1, "?");
    fprintf(file, "%-15s %-15s %-15.1f %-15s\n", "const", "Eho1        ", p.omho1 * hbar, "Energy_scale");
    fprintf(file, "%-15s %-15s %-15.6f %-15s\n", "const", "aho2        ", p.aho2, "?");
    fprintf(file, "%-15s %-15s %-15.6f %-15s\n", "const", "ax2         ", p.ax2[0], "code");
    fprintf(file, "%-15s %-15s %-15.6f %-15s\n", "const", "ay2         ", p.ax2[1], "code");
    fprintf(file, "%-15s %-15s %-15.6f %-15s\n", "const", "az2         ", p.ax2[2], "code");
    fprintf(file, "%-15s %-15s %-15.6f %-15s\n", "const", "omho2       ", p.omho2, "?");
    fprintf(file, "%-15s %-15s %-15.1f %-15s\n", "const", "Eho2        ", p.omho2 * hbar, "Energy_scale");
    fprintf(file, "%-15s %-15s %-15d %-15s\n", "const", "itmod      ", p.itmod, ".");
    fprintf(file, "%-15s %-15s %-15.6f %-15s\n", "const", "aho        ", p.aho1, "?");
    fprintf(file, "%-15s %-15s %-15.1f %-15s\n", "const", "Eho        ", p.omho1 * hbar, "Energy_scale");
    fprintf(file, "%-15s %-15s %-15.6f %-15s\n", "const", "omho       ", p.omho1, "?");
    fclose(file);
}

void Output::WriteVariable2WTXT(const char* name, double value, const char* unit) {
    FILE* file = open_or_throw(prefix + "info.wtxt", "a");
    fprintf(file, "%-15s %-15s %-15.6f %-15s\n", "const", name, value, unit);
    fclose(file);
}

void Output::WritePsi(const complex* psi, int length, const std::string& number) {
    Write3DMatrix(psi, length, number + "psi.wdat", "ab");
}
void Output::WritePsiInit(const complex* psi, int length, const std::string& number) {
    Write3DMatrix(psi, length, number + "psi_init.wdat");
}
void Output::WritePsiFinal(const complex* psi, int length, const std::string& number) {
    Write3DMatrix(psi, length, number + "psi_final.wdat");
}
void Output::WriteVext(const complex* vext, int length, const std::string& number) {
    Write3DMatrix(vext, length, number + "vext.wdat");
}

void Output::CreateStatusFile(const char* header) {
    status = open_or_throw(prefix + "status.out", "w");
    fputs(header, status);
    fflush(status);
}
void Output::WriteStatus(const char* line) {
    if (!status) status = open_or_throw(prefix + "status.out", "a");
    fputs(line, status);
    fflush(status);
}
void Output::CloseStatusFile() {
    if (status) fclose(status);
    status = nullptr;
}

void Output::Write3DMatrix(const complex* m, int length, const std::string& filename, const char* mode) {
    FILE* f = open_or_throw(prefix + filename, mode);
    size_t n = std::fwrite(m, sizeof(complex), length, f);
    std::fclose(f);
    if ((int)n != length) throw HostError("Only " + std::to_string(n) + " elements were written to " + filename);
}

}  // namespace gpe
