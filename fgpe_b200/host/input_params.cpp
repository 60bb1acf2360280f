// input_params.cpp -- input-file parser and unit conversion (host mirror).
// Same format, typing rules and arithmetic as src/input_variables.cu,
// src/params.cu and src/params2.cu, so the same input file yields bit-identical
// parameters; a missing key throws HostError instead of exit(3).
#include <cmath>
#include <fstream>
#include <iostream>
#include <sstream>

#include "gpe_host.hpp"

namespace gpe {

namespace {
std::string trim(const std::string& s) {
    size_t a = s.find_first_not_of(" \t\n\r");
    if (a == std::string::npos) return "";
    size_t b = s.find_last_not_of(" \t\n\r");
    return s.substr(a, b - a + 1);
}
bool parses_int(const std::string& s) {
    try {
        (void)std::stoi(s);
        return true;
    } catch (const std::exception&) {
        return false;
    }
}
bool parses_double(const std::string& s) {
    try {
        (void)std::stod(s);
        return true;
    } catch (const std::exception&) {
        return false;
    }
}
}  // namespace

// InputVariables::readFile / processLine, src/input_variables.cu:91-131:
// text after '#' is dropped, then the first two whitespace tokens are
// (name, value); a later line overrides an earlier one.
InputVariables::InputVariables(const std::string& filename) {
    readFile(filename);
    convertTypes();
}

void InputVariables::readFile(const std::string& filename) {
    std::ifstream file(filename);
    if (!file.is_open()) throw HostError("Error opening file: " + filename);
    std::string line;
    while (std::getline(file, line)) {
        size_t c = line.find('#');
        if (c != std::string::npos) line = line.substr(0, c);
        if (trim(line).empty()) continue;
        std::istringstream iss(line);
        std::string name, value;
        if (!(iss >> name >> value)) continue;
        variables[name] = value;
    }
}

// InputVariables::convertTypes, src/input_variables.cu:55-74: a value lands in
// every typed map whose conversion accepts it (stoi/stod accept a numeric
// prefix, so "1E-7" is both int 1 and double 1e-7).
void InputVariables::convertTypes() {
    for (const auto& e : variables) {
        if (e.second == "false" || e.second == "true") bools[e.first] = (e.second != "false");
        if (parses_int(e.second)) ints[e.first] = std::stoi(e.second);
        if (e.second.front() == '"' && e.second.back() == '"') strings[e.first] = e.second.substr(1, e.second.size() - 2);
        if (parses_double(e.second)) doubles[e.first] = std::stod(e.second);
    }
}

std::string InputVariables::getVariable(const std::string& n) const {
    auto it = variables.find(n);
    return it == variables.end() ? std::string("None") : it->second;
}
int InputVariables::getInt(const std::string& n) const {
    auto it = ints.find(n);
    if (it == ints.end()) throw HostError("Ints: No such variable " + n);
    return it->second;
}
double InputVariables::getDouble(const std::string& n) const {
    auto it = doubles.find(n);
    if (it == doubles.end()) throw HostError("Doubles: No such variable " + n);
    return it->second;
}
std::string InputVariables::getString(const std::string& n) const {
    auto it = strings.find(n);
    if (it == strings.end()) throw HostError("Strings: No such variable " + n);
    return it->second;
}
bool InputVariables::getBool(const std::string& n) const {
    auto it = bools.find(n);
    if (it == bools.end()) throw HostError("Bools: No such variable " + n);
    return it->second;
}

// Params::RedefineLatticeSoft, src/params.cu:35-131: for a soft-core droplet
// lattice the domain is made a whole number of inter-droplet distances
// idd = a_soft / (akrot / 2 pi) along each used axis, the distance scaled
// per lattice type (triangular / HEX: y by sqrt(3); BCC: sqrt(2); SC:
// 1/sqrt(2); FCC: sqrt(3)).  A missing akrot, a_soft or Latticetype key is
// an error, as in the reference (whose getDouble / getString exit before its
// try block could catch anything).  The BCC half-cell shift of the
// reference (lines 111-115) is overwritten by the plain assignment that
// follows it there, so it has no effect and is not repeated here.
void Params::redefine_lattice_soft() {
    {
        const double akrot = iv.getDouble("akrot") / (2 * pi);
        const double a = iv.getDouble("a_soft");
        const double idd = a / akrot;
        const double triangular = 2 * std::sqrt(3.) / 2.;
        double dist[3] = {idd, idd, idd};
        const std::string type = iv.getString("Latticetype");
        if (type == "triangular" || type == "HEX") dist[1] = idd * triangular;
        double f = 1.0;
        bool all = false;
        if (type == "BCC") { f = std::sqrt(2); all = true; }
        if (type == "SC") { all = true; }
        if (type == "FCC") { f = std::sqrt(3); all = true; }
        if (all)
            for (double& d : dist) d = (type == "SC") ? idd / std::sqrt(2) : idd * f;
        for (int i = 0; i < DIM && i < 3; ++i) {
            const int n = (int)std::round(2 * XMAX[i] / dist[i]);
            XMAX[i] = 0.5 * n * dist[i];
        }
    }
}

// Params::InitializeParams, src/params.cu:134-219.
Params::Params(const InputVariables& in) {
    iv = in;
    outpath = iv.getString("outprefix");
    inpath = iv.getString("inprefix");
    vpath = iv.getString("vprefix");
    NX[0] = iv.getInt("nx");
    NX[1] = iv.getInt("ny");
    NX[2] = iv.getInt("nz");
    DIM = 3;
    if (((NX[0] - 1) * (NX[1] - 1) == 1) || ((NX[1] - 1) * (NX[2] - 1) == 0)) {
        if ((NX[0] - 1) * (NX[1] - 1) == (NX[1] - 1) * (NX[2] - 1)) DIM = 1;
        else DIM = 2;
    }
    Npoints = NX[0] * NX[1] * NX[2];
    XMAX[0] = iv.getDouble("xmax");
    XMAX[1] = iv.getDouble("ymax");
    XMAX[2] = iv.getDouble("zmax");
    if (iv.has("hamiltonian") && iv.getString("hamiltonian") == "soft") redefine_lattice_soft();
    for (int i = 0; i < 3; ++i) DX[i] = 2 * XMAX[i] / NX[i];
    omega[0] = 2 * pi * iv.getDouble("omx");
    omega[1] = 2 * pi * iv.getDouble("omy");
    omega[2] = 2 * pi * iv.getDouble("omz");
    mass = iv.getDouble("mass");
    if (iv.getVariable("n1D") != "None") npart = iv.getDouble("n1D") * (2 * XMAX[0]);
    else npart = iv.getDouble("npart");
    a = iv.getDouble("a");
    if (iv.getVariable("add") != "None") {
        add = iv.getDouble("add");
        edd = add / a;
    } else {
        add = 0.0;
        edd = 0.0;
    }
    calculateLengthScales();
    dt = iv.getDouble("dt");
    time0 = iv.getDouble("time0");
    epsilon_e = iv.getDouble("epsilon_e");
    niter = iv.getInt("niter");
    itmod = iv.getInt("itmod");
    for (int i = 0; i < 3; ++i) {
        KXMAX[i] = 1.0 / (2.0 * DX[i]);
        DKX[i] = 1.0 / (NX[i] * DX[i]);
    }
    DV = DX[0] * DX[1] * DX[2];
    V = DV * Npoints;
}

// Params::calculateLengthScales, src/params.cu:223-279.
void Params::calculateLengthScales() {
    if ((std::abs(omega[0]) < 1E-6) && (std::abs(omega[1]) < 1E-6) && (std::abs(omega[2]) < 1E-6)) {
        aho = std::sqrt(hbar / (mass));
        omho = 1.0;
    } else if ((std::abs(omega[0]) < 1E-6) && (std::abs(omega[1]) < 1E-6)) {
        ax[2] = std::sqrt(hbar / (mass * omega[2]));
        aho = ax[2];
        ax[2] /= aho;
        omho = omega[2];
    } else if (std::abs(omega[0]) < 1E-6) {
        ax[1] = std::sqrt(hbar / (mass * omega[1]));
        ax[2] = std::sqrt(hbar / (mass * omega[2]));
        aho = std::sqrt(ax[1] * ax[2]);
        ax[1] /= aho;
        ax[2] /= aho;
        omho = std::sqrt(omega[2] * omega[1]);
    } else {
        for (int i = 0; i < 3; ++i) ax[i] = std::sqrt(hbar / (mass * omega[i]));
        aho = std::pow(ax[0] * ax[1] * ax[2], 1. / 3.);
        for (int i = 0; i < 3; ++i) ax[i] /= aho;
        omho = std::pow(omega[0] * omega[1] * omega[2], 1. / 3.);
    }
    a = a * abohr / aho;
    if (add != 0.0) {
        add = add * abohr / aho;
        if ((std::abs(add) < 1E-6) && (std::abs(a) < 1E-6)) edd = 0.0;
        else edd = add / a;
    }
    for (int i = 0; i < 3; ++i) {
        XMAX[i] = XMAX[i] / aho;
        DX[i] = DX[i] / aho;
    }
}

// Params2::InitializeParams, src/params2.cu:28-99 (its DIM test compares
// products with 0, so DIM stays 3 for any grid: kept).
Params2::Params2(const InputVariables& in) {
    iv = in;
    isTwoComponent = true;
    outpath = iv.getString("outprefix");
    inpath = iv.getString("inprefix");
    vpath = iv.getString("vprefix");
    NX[0] = iv.getInt("nx");
    NX[1] = iv.getInt("ny");
    NX[2] = iv.getInt("nz");
    DIM = 3;
    if ((NX[0] * NX[1] == 0) || (NX[1] * NX[2] == 0)) {
        if (NX[0] * NX[1] == NX[1] * NX[2]) DIM = 1;
        else DIM = 2;
    }
    Npoints = NX[0] * NX[1] * NX[2];
    XMAX[0] = iv.getDouble("xmax");
    XMAX[1] = iv.getDouble("ymax");
    XMAX[2] = iv.getDouble("zmax");
    for (int i = 0; i < 3; ++i) DX[i] = 2 * XMAX[i] / NX[i];
    omega1[0] = 2 * pi * iv.getDouble("omx1");
    omega1[1] = 2 * pi * iv.getDouble("omy1");
    omega1[2] = 2 * pi * iv.getDouble("omz1");
    omega2[0] = 2 * pi * iv.getDouble("omx2");
    omega2[1] = 2 * pi * iv.getDouble("omy2");
    omega2[2] = 2 * pi * iv.getDouble("omz2");
    mass1 = iv.getDouble("mass1");
    npart1 = iv.getDouble("npart1");
    a11 = iv.getDouble("a11");
    mass2 = iv.getDouble("mass2");
    npart2 = iv.getDouble("npart2");
    a22 = iv.getDouble("a22");
    a12 = iv.getDouble("a12");
    calculateLengthScales();
    dt = iv.getDouble("dt");
    time0 = iv.getDouble("time0");
    epsilon_e = iv.getDouble("epsilon_e");
    niter = iv.getInt("niter");
    itmod = iv.getInt("itmod");
    for (int i = 0; i < 3; ++i) {
        KXMAX[i] = 1.0 / (2.0 * DX[i]);
        DKX[i] = 1.0 / (NX[i] * DX[i]);
    }
    DV = DX[0] * DX[1] * DX[2];
    V = DV * Npoints;
}

// Params2::calculateLengthScales, src/params2.cu:103-186 (aho2 uses only
// ax2[1]*ax2[2] in the 3D branch, kept; different traps are rejected).
void Params2::calculateLengthScales() {
    auto scales = [](const double* om, double mass, double* ax, double& aho, double& omho, bool second) {
        if ((std::abs(om[0]) < 1E-6) && (std::abs(om[1]) < 1E-6)) {
            ax[2] = std::sqrt(hbar / (mass * om[2]));
            aho = ax[2];
            ax[2] /= aho;
            omho = om[2];
        } else if (std::abs(om[0]) < 1E-6) {
            ax[1] = std::sqrt(hbar / (mass * om[1]));
            ax[2] = std::sqrt(hbar / (mass * om[2]));
            aho = std::sqrt(ax[1] * ax[2]);
            ax[1] /= aho;
            ax[2] /= aho;
            omho = std::sqrt(om[2] * om[1]);
        } else {
            for (int i = 0; i < 3; ++i) ax[i] = std::sqrt(hbar / (mass * om[i]));
            aho = second ? std::pow(ax[1] * ax[2], 1. / 3.) : std::pow(ax[0] * ax[1] * ax[2], 1. / 3.);
            for (int i = 0; i < 3; ++i) ax[i] /= aho;
            omho = std::pow(om[0] * om[1] * om[2], 1. / 3.);
        }
    };
    scales(omega1, mass1, ax1, aho1, omho1, false);
    scales(omega2, mass2, ax2, aho2, omho2, true);
    if (std::abs(omho2 - omho1) > 1E-6)
        throw HostError("ERROR: Different traps for each spin component currently not supported.");
    a11 = a11 * abohr / aho1;
    a22 = a22 * abohr / aho1;
    a12 = a12 * abohr / aho1;
    for (int i = 0; i < 3; ++i) {
        XMAX[i] = XMAX[i] / aho1;
        DX[i] = DX[i] / aho1;
    }
}

}  // namespace gpe
