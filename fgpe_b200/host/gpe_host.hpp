// gpe_host.hpp -- host-side mirror of the reference's C++ interface (fGPE
// v0.3): input-file parser, unit conversion, initial states, output files,
// and the solver / plugin classes -- re-implemented on top of the C ABI of
// libgpe (include/gpe.h) instead of owning CUDA buffers and cuFFT plans.
//
// What is kept from the reference, so input files, plugins and output
// directories carry over unchanged:
//  - the `key value` input format and its typed maps (src/input_variables.cu)
//  - Params / Params2 fields and unit conversion (src/params.cu, src/params2.cu)
//  - Psi / Vext initialisers and .wdat readers (src/psi.cu, src/vext.cu)
//  - Output: *.wdat, info.wtxt, status.out layouts (src/output.cu)
//  - the plugin contract: alg_calcHpsi / alg_calcHpsiMU, the nine call_IM_* /
//    call_RE_* hooks, the PARS enum (hpp/oneComponentGPSolver.hpp:20-76,
//    hpp/twoComponentGPSolver.hpp:23-47)
// What differs: errors throw gpe::HostError (the reference exit()s); the
// per-iteration hooks run at the iterations where the shipped plugins act
// (every itStatMod / itmod), because the device advances whole chunks of
// steps between host round trips.
#pragma once

#include <complex>
#include <condition_variable>
#include <cstdio>
#include <deque>
#include <exception>
#include <map>
#include <mutex>
#include <random>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

#include "../../include/gpe.h"

namespace gpe {

typedef std::complex<double> complex;

// hpp/header.hpp:27-30 constants
constexpr double pi = 3.141592653589793;
constexpr double hbar = 63507.799;
constexpr double kB = (0.831466 * 1.E7);
constexpr double abohr = 5.2917721E-5;

struct HostError : std::runtime_error {
    explicit HostError(const std::string& m) : std::runtime_error(m) {}
};

// ---- src/input_variables.cu ---------------------------------------------------
class InputVariables {
public:
    InputVariables() = default;
    explicit InputVariables(const std::string& filename);
    std::string getVariable(const std::string& name) const;  // "None" when absent
    int getInt(const std::string& name) const;
    double getDouble(const std::string& name) const;
    std::string getString(const std::string& name) const;
    bool getBool(const std::string& name) const;
    bool has(const std::string& name) const { return variables.count(name) != 0; }

private:
    std::map<std::string, std::string> variables, strings;
    std::map<std::string, double> doubles;
    std::map<std::string, bool> bools;
    std::map<std::string, int> ints;
    void readFile(const std::string& filename);
    void convertTypes();
};

// ---- hpp/params.hpp, hpp/params2.hpp --------------------------------------------
class ParamsBase {
public:
    InputVariables iv;
    std::string outpath, inpath, vpath;
    bool isTwoComponent = false;
    int NX[3] = {0, 0, 0};
    int DIM = 3;
    int Npoints = 0;
    double V = 0, XMAX[3] = {0, 0, 0}, DX[3] = {0, 0, 0}, DV = 0;
    double KXMAX[3] = {0, 0, 0}, DKX[3] = {0, 0, 0};
    double dt = 0, epsilon_e = 0, time0 = 0;
    int niter = 0, itmod = 1;

    virtual ~ParamsBase() = default;
    virtual const double* _omega(int type) const = 0;
    virtual const double* _ax(int type) const = 0;
    virtual double _aho(int type) const = 0;
    virtual double _omho(int type) const = 0;
    virtual double _npart(int type) const = 0;
    int getInt(const std::string& n) const { return iv.getInt(n); }
    double getDouble(const std::string& n) const { return iv.getDouble(n); }
    std::string getString(const std::string& n) const { return iv.getString(n); }
    bool getBool(const std::string& n) const { return iv.getBool(n); }
    const InputVariables& getIV() const { return iv; }
};

class Params : public ParamsBase {
public:
    double omega[3] = {0, 0, 0}, ax[3] = {0, 0, 0};
    double aho = 0, omho = 0, mass = 0, npart = 0, a = 0, add = 0, edd = 0;
    Params() = default;
    explicit Params(const InputVariables& iv);
    // Params::RedefineLatticeSoft (src/params.cu:35-131), applied for
    // hamiltonian "soft" before DX is derived from XMAX.
    void redefine_lattice_soft();
    const double* _omega(int) const override { return omega; }
    const double* _ax(int) const override { return ax; }
    double _aho(int) const override { return aho; }
    double _omho(int) const override { return omho; }
    double _npart(int) const override { return npart; }

private:
    void calculateLengthScales();
};

class Params2 : public ParamsBase {
public:
    double omega1[3] = {0, 0, 0}, omega2[3] = {0, 0, 0}, ax1[3] = {0, 0, 0}, ax2[3] = {0, 0, 0};
    double aho1 = 0, omho1 = 0, aho2 = 0, omho2 = 0;
    double mass1 = 0, mass2 = 0, npart1 = 0, npart2 = 0, a11 = 0, a22 = 0, a12 = 0;
    Params2() = default;
    explicit Params2(const InputVariables& iv);
    const double* _omega(int t) const override { return t == 1 ? omega1 : omega2; }
    const double* _ax(int t) const override { return t == 1 ? ax1 : ax2; }
    double _aho(int t) const override { return t == 1 ? aho1 : aho2; }
    double _omho(int t) const override { return t == 1 ? omho1 : omho2; }
    double _npart(int t) const override { return t == 1 ? npart1 : npart2; }

private:
    void calculateLengthScales();
};

// ---- hpp/psi.hpp, hpp/vext.hpp -------------------------------------------------
// Grid positions (cell centred), src/psi.cu:134-150.
double gridX(const ParamsBase& p, int i);
double gridY(const ParamsBase& p, int i);
double gridZ(const ParamsBase& p, int i);

class Psi {
public:
    std::vector<complex> psi;
    Psi(const Params& p, const std::string& type);  // 1 component (src/psi.cu:7-32)
    Psi(const ParamsBase& p, int type);             // component type of 2 (src/psi.cu:50-77)
    void initTube(const ParamsBase& p, int type);
    void initHarmonic(const ParamsBase& p, int type);
    void normalize(const ParamsBase& p, int type = -1);
    void imprintVortexTube(const ParamsBase& p, double Ncirc);
    // Lattice seeds for soft-core droplet crystals (src/psi.cu:179-348): add
    // amp * (a sum of plane-wave cosines of wave number k, offset by off*)
    // times sqrt(npart / dV) to psi, then normalise to the first component's
    // particle number (the reference always passes 1 there).
    void force1DLattice(const ParamsBase& p, double amp, double k, double off, int type = 1);
    void force2DTriangularLattice(const ParamsBase& p, double amp, double k, double offx, double offy, int type = 1);
    void force2DSquareLattice(const ParamsBase& p, double amp, double k, double offx, double offy, int type = 1);
    void force3DHEXLattice(const ParamsBase& p, double amp, double k, double offx, double offy, double offz,
                           int type = 1);
    void force3DFCCLattice(const ParamsBase& p, double amp, double k, double offx, double offy, double offz,
                           int type = 1);
    void force3DBCCLattice(const ParamsBase& p, double amp, double k, double offx, double offy, double offz,
                           int type = 1);
    void force3DSCLattice(const ParamsBase& p, double amp, double k, double offx, double offy, double offz,
                          int type = 1);
    void readPsi(const std::string& prefix, int length);
    complex* getPsi() { return psi.data(); }

private:
    template <class Shape>
    void add_lattice(const ParamsBase& p, int type, Shape shape);
    std::mt19937 generator;
    std::uniform_real_distribution<double> distribution{-1.0, 1.0};
    complex noise(double rrnd, double crnd);
};

class Vext {
public:
    std::vector<complex> vext;
    Vext(const Params& p, const std::string& type);
    Vext(const Params2& p, int type);
    void initTube(const ParamsBase& p, int type);
    void initHarmonic(const ParamsBase& p, int type);
    void readVext(const std::string& prefix, int length);
    void addProtocolPotential(const ParamsBase& p, int type, int sign = 1);
    void addWeightedProtocolPotential(const Params2& p, int type);
    complex* getVext() { return vext.data(); }
};

// ---- hpp/output.hpp -------------------------------------------------------------
class Output {
public:
    explicit Output(const std::string& prefix) : prefix(prefix) {}
    void WriteWtxt(const Params& p, int ncycle);
    void WriteWtxt_2c(const Params2& p, int ncycle);
    void WriteVariable2WTXT(const char* name, double value, const char* unit);
    void WritePsi(const complex* psi, int length, const std::string& number = "");
    void WritePsiInit(const complex* psi, int length, const std::string& number = "");
    void WritePsiFinal(const complex* psi, int length, const std::string& number = "");
    void WriteVext(const complex* vext, int length, const std::string& number = "");
    void CreateStatusFile(const char* header);
    void WriteStatus(const char* line);
    void CloseStatusFile();
    void Write3DMatrix(const complex* m, int length, const std::string& filename, const char* mode = "wb");
    const std::string& getPrefix() const { return prefix; }

private:
    std::string prefix;
    FILE* status = nullptr;
};

// Asynchronous psi.wdat frame appends (frame_writer.cpp): push(suffixes)
// queues the solver's current psi (all components) -- converted to
// complex128 on the device and copied into one of two pinned host slots on
// the default stream the solver's handle runs on -- and a writer thread
// appends component c to <prefix><suffixes[c]>psi.wdat once the copy has
// landed, so stepping continues while the files are written.  Frames reach
// the files in push order; push() waits only when both slots are still being
// written.  flush() returns when every queued frame is on disk and rethrows
// a write error.
class FrameWriter {
public:
    FrameWriter() = default;
    FrameWriter(const FrameWriter&) = delete;
    FrameWriter& operator=(const FrameWriter&) = delete;
    ~FrameWriter();
    bool started() const { return out_ != nullptr; }
    void start(Output* out, gpe_handle* h, long long n, int ncomp);
    void push(const std::vector<std::string>& suffixes);
    void flush();

private:
    struct Frame {
        int slot;
        std::vector<std::string> suffixes;
    };
    void run();
    Output* out_ = nullptr;
    gpe_handle* h_ = nullptr;
    long long n_ = 0;
    int ncomp_ = 0;
    void* dev_ = nullptr;
    void* host_[2] = {nullptr, nullptr};
    void* ev_[2] = {nullptr, nullptr};  // cudaEvent_t
    bool busy_[2] = {false, false};
    int slot_ = 0;
    std::deque<Frame> queue_;
    bool stop_ = false;
    std::exception_ptr err_;
    std::mutex m_;
    std::condition_variable cv_;
    std::thread thread_;
};

// ---- solver / plugin classes ------------------------------------------------------
// Mirrors OneComponentGPSolver (src/oneComponentGPSolver.cu) over a libgpe handle.
class OneComponentGPSolver {
public:
    Params p;
    Output output;
    std::vector<complex> psi, vext;
    gpe_handle* h = nullptr;
    double PARS[32] = {0.0};
    enum Variables { T, EN, MU, NORM, PX, LZ, EN_PREV, AVG_TIME, ITER, ITER_TIME, EN_0, MU_0, NCYCLES,
                     AUX1, AUX2, AUX3, AUX4, AUX5 };

    explicit OneComponentGPSolver(const Params& par, int hamiltonian);
    virtual ~OneComponentGPSolver();
    void runImagTimeEvol();
    void runRealTimeEvol();
    // Hamiltonian parameters d_h_params (hamiltonians/BEC_oneComponent.cu:10-15).
    void setHamiltonianParams(const double* prms);
    // Plugin contract: h of the current psi (both / mu only) into host arrays.
    virtual void alg_calcHpsi(std::vector<complex>* hmu, std::vector<complex>* hen);
    virtual void alg_calcHpsiMU(std::vector<complex>* hmu);
    virtual void call_IM_init() {}
    virtual void call_IM_loop_before_step() {}
    virtual void call_IM_loop_after_step() {}
    virtual void call_IM_loop_convergence() {}
    virtual void call_IM_end() {}
    virtual void call_RE_init() {}
    virtual void call_RE_loop_before_step() {}
    virtual void call_RE_loop_after_step() {}
    virtual void call_RE_end() {}
    void download_psi();
    // Appends the current psi to psi.wdat without stopping the stepping loop
    // (a plugin's replacement for download_psi() + output.WritePsi(psi)).
    void write_frame();
    int itStatMod() const;
    // raw norm / <psi|h_mu> / <psi|h_en> sums of the last status step
    double last_obs[6] = {0, 0, 0, 0, 0, 0};

protected:
    gpe_config make_config(int hamiltonian) const;
    FrameWriter frames;  // last member: destroyed (flushed) before output and h
};

class TwoComponentGPSolver {
public:
    Params2 p;
    Output output;
    std::vector<complex> psi1, psi2, vext1, vext2;
    gpe_handle* h = nullptr;
    double PARS[64] = {0.0};
    enum Variables { EN1, EN2, MU1, MU2, NORM1, NORM2, PX1, PX2, EN1_PREV, EN2_PREV, AVG_TIME, ITER, ITER_TIME,
                     EN1_0, EN2_0, MU1_0, MU2_0, NCYCLES, AUX1_1, AUX2_1, AUX3_1, AUX4_1, AUX5_1, AUX1_2, AUX2_2,
                     AUX3_2, AUX4_2, AUX5_2 };

    explicit TwoComponentGPSolver(const Params2& par);
    virtual ~TwoComponentGPSolver();
    void runImagTimeEvol();
    void runRealTimeEvol();
    virtual void call_IM_init() {}
    virtual void call_IM_loop_after_step() {}
    virtual void call_IM_loop_convergence() {}
    virtual void call_IM_end() {}
    virtual void call_RE_init() {}
    virtual void call_RE_loop_after_step() {}
    virtual void call_RE_end() {}
    void download_psi();
    // Appends psi1 and psi2 to <suffix1>psi.wdat and <suffix2>psi.wdat without
    // stopping the stepping loop (replaces download_psi() + two WritePsi calls).
    void write_frames(const std::string& suffix1, const std::string& suffix2);
    void upload();
    int itStatMod() const;

protected:
    FrameWriter frames;  // last member: destroyed (flushed) before output and h
};

// hamiltonians/BEC_oneComponent.{hpp,cu}
class BEConeComponent : public OneComponentGPSolver {
public:
    explicit BEConeComponent(const Params& par, bool run = true, int hamiltonian = GPE_HAM_BEC);
    void InitPsi();
    void InitVext();
    void call_IM_init() override;
    void call_IM_loop_after_step() override;
    void call_IM_loop_convergence() override;
    void call_IM_end() override;
    void call_RE_init() override;
    void call_RE_loop_after_step() override;
    void call_RE_end() override;
    double calcPx();
    bool is_template = false;
};

// hamiltonians/single_template.{hpp,cu}: h = T only.
class SingleTemplate : public BEConeComponent {
public:
    explicit SingleTemplate(const Params& par, bool run = true);
};

// hamiltonians/BEC_twoComponent.{hpp,cu}
class BECtwoComponent : public TwoComponentGPSolver {
public:
    explicit BECtwoComponent(const Params2& par, bool run = true);
    void InitPsi();
    void InitVext();
    void call_IM_init() override;
    void call_IM_loop_after_step() override;
    void call_IM_loop_convergence() override;
    void call_IM_end() override;
    void call_RE_init() override;
    void call_RE_loop_after_step() override;
    void call_RE_end() override;
    double calcPx(int comp);
    void status_line_imag();
    void status_line_real(double time);
};

// main.cu:20-82: run an input file; returns a process exit code.
int run_input_file(const std::string& file);

}  // namespace gpe
