// solvers.cpp -- solver and plugin classes of the host mirror, driving libgpe.
//
// The loops follow OneComponentGPSolver::runImagTimeEvol / runRealTimeEvol
// (src/oneComponentGPSolver.cu:26-217) and TwoComponentGPSolver's
// (src/twoComponentGPSolver.cu:15-209), but advance the device a chunk of
// iterations per C-ABI call: a chunk ends at the next iteration whose hook
// acts (a status line every itStatMod, a psi frame every itmod) or at
// convergence, which the device detects itself.  The hooks of the shipped
// plugins (hamiltonians/BEC_oneComponent.cu:197-400,
// hamiltonians/BEC_twoComponent.cu:267-493) write the same files.
#include <chrono>
#include <cmath>
#include <cstring>
#include <iostream>

#include "gpe_host.hpp"

namespace gpe {

namespace {

void chk(gpe_status s, const char* what) {
    if (s != GPE_OK) throw HostError(std::string(what) + ": " + gpe_last_error_string());
}

double now_ms() {
    using namespace std::chrono;
    return duration<double, std::milli>(steady_clock::now().time_since_epoch()).count();
}

// Keys that exist only in this build: `precision` ("c128" default, "c64") and
// `imag_scheme` ("heavyball" default, "rk4").
int precision_from(const ParamsBase& p) {
    const std::string v = p.getIV().getVariable("precision");
    if (v == "None" || v == "\"c128\"") return GPE_C128;
    if (v == "\"c64\"") return GPE_C64;
    throw HostError("precision must be \"c128\" or \"c64\"");
}
int scheme_from(const ParamsBase& p) {
    const std::string v = p.getIV().getVariable("imag_scheme");
    if (v == "None" || v == "\"heavyball\"") return GPE_IMAG_HEAVYBALL;
    if (v == "\"rk4\"") return GPE_IMAG_RK4;
    throw HostError("imag_scheme must be \"heavyball\" or \"rk4\"");
}
double opt_double(const ParamsBase& p, const char* key, double dflt) {
    return p.getIV().getVariable(key) != "None" ? p.getDouble(key) : dflt;
}

void fill_grid(gpe_config& c, const ParamsBase& p) {
    c.nx = p.NX[0];
    c.ny = p.NX[1];
    c.nz = p.NX[2];
    c.dim = p.DIM;
    for (int d = 0; d < 3; ++d) {
        c.xmax[d] = p.XMAX[d];
        c.dx[d] = p.DX[d];
    }
    c.precision = precision_from(p);
    c.imag_scheme = scheme_from(p);
    c.epsilon_e = p.epsilon_e;
    c.beta = opt_double(p, "beta", 0.0);
}

// <cos(2 pi x / L)>: CalcAverageCos, src/parallel.cu:535-561, times DV.
// First iteration i >= it (at most last) for which pred(i) holds.
template <class Pred>
int next_event(int it, int last, Pred pred) {
    int i = it;
    while (i < last && !pred(i)) ++i;
    return i;
}

}  // namespace

// ==== one component ====================================================================
gpe_config OneComponentGPSolver::make_config(int hamiltonian) const {
    gpe_config c;
    gpe_config_init(&c);
    fill_grid(c, p);
    c.ncomp = 1;
    c.hamiltonian = hamiltonian;
    c.dt = p.dt * p.omho / 1000;  // src/oneComponentGPSolver.cu:39,134
    c.npart[0] = p.npart;
    return c;
}

OneComponentGPSolver::OneComponentGPSolver(const Params& par, int hamiltonian) : p(par), output(par.outpath) {
    psi.assign(p.Npoints, complex(0, 0));
    vext.assign(p.Npoints, complex(0, 0));
    gpe_config c = make_config(hamiltonian);
    chk(gpe_create(&c, &h), "gpe_create");
}

OneComponentGPSolver::~OneComponentGPSolver() {
    try {
        frames.flush();
    } catch (...) {
    }
    if (h) gpe_destroy(h);
}

void OneComponentGPSolver::setHamiltonianParams(const double* prms) { chk(gpe_set_params(h, prms), "gpe_set_params"); }

int OneComponentGPSolver::itStatMod() const { return p.getInt("itStatMod"); }

void OneComponentGPSolver::download_psi() { chk(gpe_get_psi(h, 0, (double*)psi.data()), "gpe_get_psi"); }

void OneComponentGPSolver::write_frame() {
    if (!frames.started()) frames.start(&output, h, p.Npoints, 1);
    frames.push({""});
}

void OneComponentGPSolver::alg_calcHpsi(std::vector<complex>* hmu, std::vector<complex>* hen) {
    if (hmu) hmu->resize(p.Npoints);
    if (hen) hen->resize(p.Npoints);
    chk(gpe_apply_h(h, PARS[T], 0, hmu ? (double*)hmu->data() : nullptr, hen ? (double*)hen->data() : nullptr),
        "gpe_apply_h");
}

void OneComponentGPSolver::alg_calcHpsiMU(std::vector<complex>* hmu) { alg_calcHpsi(hmu, nullptr); }

void OneComponentGPSolver::runImagTimeEvol() {
    call_IM_init();
    chk(gpe_set_vext(h, 0, (const double*)vext.data()), "gpe_set_vext");
    chk(gpe_set_psi(h, 0, (const double*)psi.data()), "gpe_set_psi");
    const int sm = itStatMod(), im = p.itmod;
    int it = 0;
    while (it < p.niter) {
        const int nxt = next_event(it, p.niter - 1, [&](int i) { return i % sm == 0 || (i + 1) % im == 0; });
        const double t0 = now_ms();
        int done = 0, conv = 0;
        call_IM_loop_before_step();
        chk(gpe_step_imag(h, it, nxt - it + 1, &done, &conv), "gpe_step_imag");
        const double el = now_ms() - t0;
        PARS[AVG_TIME] += el;
        PARS[ITER_TIME] = el / (done > 0 ? done : 1);
        double st[4];
        chk(gpe_imag_state(h, st), "gpe_imag_state");
        PARS[NORM] = st[0];
        PARS[MU] = st[1];
        PARS[EN] = st[2];
        PARS[EN_PREV] = st[3];
        if (conv) {
            PARS[ITER] = it + done - 1;
            call_IM_loop_convergence();
            break;
        }
        PARS[ITER] = nxt;
        call_IM_loop_after_step();
        PARS[ITER] = nxt + 1;
        it = nxt + 1;
    }
    frames.flush();
    download_psi();
    call_IM_end();
}

void OneComponentGPSolver::runRealTimeEvol() {
    chk(gpe_set_vext(h, 0, (const double*)vext.data()), "gpe_set_vext");
    chk(gpe_set_psi(h, 0, (const double*)psi.data()), "gpe_set_psi");
    const double dt = p.dt * p.omho / 1000;
    call_RE_init();
    PARS[T] = 0;
    PARS[AVG_TIME] = 0;
    const int sm = itStatMod(), im = p.itmod;
    int it = 0;
    while (it < p.niter) {
        // PARS[ITER] = iteration+1 inside the hooks (src/oneComponentGPSolver.cu:156)
        const int nxt = next_event(it, p.niter - 1, [&](int i) { return (i + 1) % sm == 0 || (i + 2) % im == 0; });
        const bool status = ((nxt + 1) % sm == 0);
        call_RE_loop_before_step();
        const double t0 = now_ms();
        chk(gpe_step_real(h, it, nxt - it + 1, status ? last_obs : nullptr), "gpe_step_real");
        if (!status) chk(gpe_sync(h), "gpe_sync");
        const double el = now_ms() - t0;
        PARS[AVG_TIME] += el;
        PARS[ITER_TIME] = el / (nxt - it + 1);
        PARS[ITER] = nxt + 1;
        PARS[T] = (nxt + 1) * dt;
        call_RE_loop_after_step();
        it = nxt + 1;
    }
    frames.flush();
    download_psi();
    call_RE_end();
}

// ==== BEC one component (hamiltonians/BEC_oneComponent.cu) ===========================
BEConeComponent::BEConeComponent(const Params& par, bool run, int hamiltonian)
    : OneComponentGPSolver(par, hamiltonian) {
    is_template = (hamiltonian == GPE_HAM_TEMPLATE);
    InitPsi();
    InitVext();
    double hp[GPE_NO_HAMIL_PARAMS] = {0};
    // hamiltonians/BEC_oneComponent.cu:14: only a is set, so d_quench_as
    // returns prms[2] = 0 and the shipped "bec" plugin runs with g = 0.  The
    // optional quench_* keys fill prms[0..5] (a0,a1,a2 = a*f0..2; t1..t3).
    hp[0] = p.a;
    const bool quench = p.getIV().getVariable("quench_f0") != "None" ||
                        p.getIV().getVariable("quench_f1") != "None" ||
                        p.getIV().getVariable("quench_f2") != "None" || hamiltonian == GPE_HAM_DIPOLAR;
    if (quench) {
        hp[0] = p.a * opt_double(p, "quench_f0", 1.0);
        hp[1] = p.a * opt_double(p, "quench_f1", 1.0);
        hp[2] = p.a * opt_double(p, "quench_f2", 1.0);
        hp[3] = opt_double(p, "quench_t1", 0.0);
        hp[4] = opt_double(p, "quench_t2", 0.0);
        hp[5] = opt_double(p, "quench_t3", 0.0);
    }
    if (hamiltonian == GPE_HAM_DIPOLAR) {
        hp[6] = p.add;
        hp[7] = opt_double(p, "dipole_x", 0.0);
        hp[8] = opt_double(p, "dipole_y", 0.0);
        hp[9] = opt_double(p, "dipole_z", 1.0);
        hp[10] = opt_double(p, "rcutoff", 0.0) / p.aho;  // same length unit as xmax
    }
    // hamiltonians/BEC_oneComponent.cu:98-101: trotate adds alg_addVPx with
    // lambda = 2 pi omega / (omho aho) (the template plugin has no such term)
    if (!is_template && p.getBool("trotate")) hp[11] = 2 * pi * p.getDouble("omega") / (p.omho * p.aho);
    setHamiltonianParams(hp);
    if (!run) return;
    if (p.getBool("treal")) {
        std::cout << "# Running real time evolution" << std::endl;
        runRealTimeEvol();
    } else {
        std::cout << "# Running imaginary time evolution" << std::endl;
        runImagTimeEvol();
    }
}

void BEConeComponent::InitPsi() {
    Psi ps(p, std::string(""));
    if (p.getBool("tpi_vortex")) ps.imprintVortexTube(p, p.getDouble("api_prc"));
    if (!is_template) output.WritePsiInit(ps.getPsi(), p.Npoints);
    psi = ps.psi;
}

void BEConeComponent::InitVext() {
    Vext v(p, std::string(""));
    if (!is_template && p.getBool("tvseed")) v.addProtocolPotential(p, 0);
    if (!is_template) output.WriteVext(v.getVext(), p.Npoints);
    vext = v.vext;
}

double BEConeComponent::calcPx() {
    double px = 0;
    chk(gpe_momentum_x(h, 0, &px), "gpe_momentum_x");
    return px;
}

void BEConeComponent::call_IM_init() {
    char buf[256];
    snprintf(buf, sizeof buf, "%-7s %-10s %-10s %-15s %-15s %-10s %-15s\n", "Iter.", "Time", "Norm", "mu", "Energy",
             "Ediff", "<Px>");
    output.CreateStatusFile(buf);
    output.WritePsiInit(psi.data(), p.Npoints);
}

void BEConeComponent::call_IM_loop_after_step() {
    char buf[256];
    const int iteration = (int)PARS[ITER];
    if (iteration % itStatMod() == 0) {
        PARS[PX] = calcPx();
        PARS[PX] /= PARS[NORM] / p.aho;
        snprintf(buf, sizeof buf, "%-7d %-10.4f %-10.1f %-15.12f %-15.12f %-10.3E %-15.12f\n", (int)PARS[ITER],
                 PARS[ITER_TIME], PARS[NORM], PARS[MU], PARS[EN], PARS[EN_PREV] - PARS[EN], PARS[PX] / hbar);
        output.WriteStatus(buf);
    }
    if ((iteration + 1) % p.itmod == 0) write_frame();
}

void BEConeComponent::call_IM_loop_convergence() {
    char buf[256];
    PARS[PX] = calcPx();
    if (is_template) {
        PARS[PX] /= PARS[NORM] / p.aho;
        snprintf(buf, sizeof buf, "%-7d %-10.4f %-10.1f %-15.12f %-15.12f %-10.3E %-15.12f\n", (int)PARS[ITER],
                 PARS[ITER_TIME], PARS[NORM], PARS[MU], PARS[EN], PARS[EN_PREV] - PARS[EN], PARS[PX] / hbar);
    } else {
        PARS[PX] /= PARS[NORM] / p.aho * hbar;  // hamiltonians/BEC_oneComponent.cu:253
        snprintf(buf, sizeof buf, "%-7d %-10.4f %-10.1f %-15.12f %-15.12f %-10.3E %-15.12f\n", (int)PARS[ITER],
                 PARS[ITER_TIME], PARS[NORM], PARS[MU], PARS[EN], PARS[EN_PREV] - PARS[EN], PARS[PX]);
    }
    output.WriteStatus(buf);
    std::cout << "Convergence reached: dE = " << PARS[EN_PREV] - PARS[EN] << std::endl;
}

void BEConeComponent::call_IM_end() {
    output.WritePsiFinal(psi.data(), p.Npoints);
    output.CloseStatusFile();
    output.WriteWtxt(p, 1);
    output.WriteVariable2WTXT("en", PARS[EN], "code");
    output.WriteVariable2WTXT("mu", PARS[MU], "code");
    output.WriteVariable2WTXT("px", PARS[PX], "hbar");
    output.WriteVariable2WTXT("convergence", PARS[EN_PREV] - PARS[EN], "code");
    std::cout << "Average iteration time: " << PARS[AVG_TIME] / PARS[ITER] << std::endl;
    std::cout << "Files saved under prefix: " << p.outpath << std::endl;
}

void BEConeComponent::call_RE_init() {
    char buf[256];
    snprintf(buf, sizeof buf, "%-15s %-10s %-10s %-15s %-15s %-15s %-15s %-10s\n", "Time", "ItTime", "Norm", "mu",
             "Energy", "Px", "<cos>", "Ediff");
    output.CreateStatusFile(buf);
    output.WritePsiInit(psi.data(), p.Npoints);
    PARS[NORM] = p.npart;
    // alg_calcHpsi + alg_calc2Observables(npart) + alg_calcNorm
    // (hamiltonians/BEC_oneComponent.cu:318-320)
    double o[6];
    chk(gpe_observables(h, 0.0, o), "gpe_observables");
    PARS[MU_0] = o[1] / PARS[NORM];
    PARS[EN_0] = o[2] / PARS[NORM];
    PARS[NORM] = o[0];
    if (!is_template) {
        chk(gpe_average_cos(h, 0, &PARS[AUX1]), "gpe_average_cos");  // alg_calcCos on the device
        PARS[AUX1] /= PARS[NORM];
    }
    PARS[PX] = calcPx();
    PARS[PX] /= (PARS[NORM] * hbar) / p.aho;
    snprintf(buf, sizeof buf, "%-15.5f %-10.4f %-10.1f %-15.12f %-15.12f %-15.12f %-15.12f %-10.3E\n", 0.0, 0.0,
             PARS[NORM], PARS[MU_0], PARS[EN_0], PARS[PX], PARS[AUX1], PARS[EN_0] - PARS[EN]);
    output.WriteStatus(buf);
}

void BEConeComponent::call_RE_loop_after_step() {
    char buf[256];
    if (((int)PARS[ITER]) % itStatMod() == 0) {
        // alg_calcNorm + alg_calc2Observables with H of the last stage argument
        // (hamiltonians/BEC_oneComponent.cu:347-348), reduced by the device
        // during the last step of the chunk.
        PARS[NORM] = last_obs[0];
        PARS[MU] = last_obs[1] / PARS[NORM];
        PARS[EN] = last_obs[2] / PARS[NORM];
        if (!is_template) {
            chk(gpe_average_cos(h, 0, &PARS[AUX1]), "gpe_average_cos");
            PARS[AUX1] /= PARS[NORM];
        }
        PARS[PX] = calcPx();
        PARS[PX] /= (PARS[NORM] * hbar) / p.aho;
        const double time = p.time0 + PARS[ITER] * p.dt;
        snprintf(buf, sizeof buf, "%-15.5f %-10.4f %-10.1f %-15.12f %-15.12f %-15.12f %-15.12f %-10.3E\n", time,
                 PARS[ITER_TIME], PARS[NORM], PARS[MU], PARS[EN], PARS[PX], PARS[AUX1], PARS[EN] - PARS[EN_0]);
        output.WriteStatus(buf);
    }
    if (((int)PARS[ITER] + 1) % p.itmod == 0) {
        write_frame();
        PARS[NCYCLES]++;
    }
}

void BEConeComponent::call_RE_end() {
    output.WritePsiFinal(psi.data(), p.Npoints);
    output.CloseStatusFile();
    output.WriteWtxt(p, (int)PARS[NCYCLES]);
    output.WriteVariable2WTXT("en0", PARS[EN_0], "code");
    output.WriteVariable2WTXT("mu0", PARS[MU_0], "code");
    output.WriteVariable2WTXT("en", PARS[EN], "code");
    output.WriteVariable2WTXT("mu", PARS[MU_0], "code");  // the reference writes MU_0 here
    output.WriteVariable2WTXT("px", PARS[PX], "hbar");
    std::cout << "Average iteration time: " << PARS[AVG_TIME] / PARS[ITER] << std::endl;
    std::cout << "Files saved under prefix: " << p.outpath << std::endl;
}

SingleTemplate::SingleTemplate(const Params& par, bool run) : BEConeComponent(par, run, GPE_HAM_TEMPLATE) {}

// ==== two components =====================================================================
TwoComponentGPSolver::TwoComponentGPSolver(const Params2& par) : p(par), output(par.outpath) {
    psi1.assign(p.Npoints, complex(0, 0));
    psi2 = vext1 = vext2 = psi1;
    gpe_config c;
    gpe_config_init(&c);
    fill_grid(c, p);
    c.ncomp = 2;
    c.hamiltonian = GPE_HAM_BEC2;
    c.dt = p.dt * p.omho1 / 1000;  // src/twoComponentGPSolver.cu:32
    c.npart[0] = p.npart1;
    c.npart[1] = p.npart2;
    chk(gpe_create(&c, &h), "gpe_create");
}

TwoComponentGPSolver::~TwoComponentGPSolver() {
    try {
        frames.flush();
    } catch (...) {
    }
    if (h) gpe_destroy(h);
}

void TwoComponentGPSolver::write_frames(const std::string& suffix1, const std::string& suffix2) {
    if (!frames.started()) frames.start(&output, h, p.Npoints, 2);
    frames.push({suffix1, suffix2});
}

int TwoComponentGPSolver::itStatMod() const { return p.getInt("itStatMod"); }

void TwoComponentGPSolver::download_psi() {
    chk(gpe_get_psi(h, 0, (double*)psi1.data()), "gpe_get_psi");
    chk(gpe_get_psi(h, 1, (double*)psi2.data()), "gpe_get_psi");
}

void TwoComponentGPSolver::upload() {
    chk(gpe_set_vext(h, 0, (const double*)vext1.data()), "gpe_set_vext");
    chk(gpe_set_vext(h, 1, (const double*)vext2.data()), "gpe_set_vext");
    chk(gpe_set_psi(h, 0, (const double*)psi1.data()), "gpe_set_psi");
    chk(gpe_set_psi(h, 1, (const double*)psi2.data()), "gpe_set_psi");
}

void TwoComponentGPSolver::runImagTimeEvol() {
    call_IM_init();
    upload();
    const int sm = itStatMod(), im = p.itmod;
    int it = 0;
    while (it < p.niter) {
        const int nxt = next_event(it, p.niter - 1, [&](int i) { return i % sm == 0 || (i + 1) % im == 0; });
        const double t0 = now_ms();
        int done = 0, conv = 0;
        chk(gpe_step_imag(h, it, nxt - it + 1, &done, &conv), "gpe_step_imag");
        const double el = now_ms() - t0;
        PARS[AVG_TIME] += el;
        PARS[ITER_TIME] = el / (done > 0 ? done : 1);
        double st[8];
        chk(gpe_imag_state(h, st), "gpe_imag_state");
        PARS[NORM1] = st[0];
        PARS[MU1] = st[1];
        PARS[EN1] = st[2];
        PARS[EN1_PREV] = st[3];
        PARS[NORM2] = st[4];
        PARS[MU2] = st[5];
        PARS[EN2] = st[6];
        PARS[EN2_PREV] = st[7];
        if (conv) {
            PARS[ITER] = it + done - 1;
            call_IM_loop_convergence();
            break;
        }
        PARS[ITER] = nxt;
        call_IM_loop_after_step();
        PARS[ITER] = nxt + 1;
        it = nxt + 1;
    }
    frames.flush();
    download_psi();
    call_IM_end();
}

// src/twoComponentGPSolver.cu:120-209: the loop starts at iteration = 1, so
// niter-1 steps run; PARS[ITER] is incremented after each step's hook.
void TwoComponentGPSolver::runRealTimeEvol() {
    upload();
    call_RE_init();
    const int sm = itStatMod(), im = p.itmod;
    int it = 1;
    while (it < p.niter) {
        const int base = (int)PARS[ITER] - it;  // PARS[ITER] = it + base inside the hook
        const int nxt = next_event(it, p.niter - 1,
                                   [&](int i) { return (i + base) % sm == 0 || (i + base + 1) % im == 0; });
        const double t0 = now_ms();
        chk(gpe_step_real(h, it, nxt - it + 1, nullptr), "gpe_step_real");
        chk(gpe_sync(h), "gpe_sync");
        const double el = now_ms() - t0;
        PARS[AVG_TIME] += el;
        PARS[ITER_TIME] = el / (nxt - it + 1);
        PARS[ITER] = nxt + base;
        call_RE_loop_after_step();
        PARS[ITER] = nxt + base + 1;
        it = nxt + 1;
    }
    frames.flush();
    download_psi();
    call_RE_end();
}

// ==== BEC two components (hamiltonians/BEC_twoComponent.cu) ===============================
BECtwoComponent::BECtwoComponent(const Params2& par, bool run) : TwoComponentGPSolver(par) {
    InitPsi();
    InitVext();
    double hp[GPE_NO_HAMIL_PARAMS] = {0};
    hp[0] = p.a11;
    hp[1] = p.a22;
    hp[2] = p.a12;
    // hamiltonians/BEC_twoComponent.cu:125-129: trotate adds alg_addVPx with
    // lambda = 2 pi omega / (omho aho) per component
    if (p.getBool("trotate")) {
        hp[11] = 2 * pi * p.getDouble("omega") / (p.omho1 * p.aho1);
        hp[12] = 2 * pi * p.getDouble("omega") / (p.omho2 * p.aho2);
    }
    chk(gpe_set_params(h, hp), "gpe_set_params");
    if (!run) return;
    if (p.getBool("treal")) {
        std::cout << "# Running real time evolution" << std::endl;
        runRealTimeEvol();
    } else {
        std::cout << "# Running imaginary time evolution" << std::endl;
        runImagTimeEvol();
    }
}

void BECtwoComponent::InitPsi() {
    Psi p1(p, 1), p2(p, 2);
    if (p.getBool("tpi_vortex")) {
        p1.imprintVortexTube(p, p.getDouble("api_prc"));
        p2.imprintVortexTube(p, p.getDouble("api_prc"));
    }
    psi1 = p1.psi;
    psi2 = p2.psi;
}

void BECtwoComponent::InitVext() {
    Vext v1(p, 1), v2(p, 2);
    if (p.getBool("tvseed")) {
        v1.addWeightedProtocolPotential(p, 1);
        v2.addWeightedProtocolPotential(p, 2);
    }
    output.WriteVext(v1.getVext(), p.Npoints, "1");
    output.WriteVext(v2.getVext(), p.Npoints, "2");
    vext1 = v1.vext;
    vext2 = v2.vext;
}

double BECtwoComponent::calcPx(int comp) {
    double px = 0;
    chk(gpe_momentum_x(h, comp, &px), "gpe_momentum_x");
    return px;
}

void BECtwoComponent::status_line_imag() {
    char buf[320];
    snprintf(buf, sizeof buf,
             "%-7d %-10.4f %-10.1f %-15.12f %-15.12f %-15.12f %-10.1f %-15.12f %-15.12f %-15.12f %-10.3E %-10.3E\n",
             (int)PARS[ITER], PARS[ITER_TIME], PARS[NORM1], PARS[MU1], PARS[EN1], PARS[PX1] / hbar, PARS[NORM2],
             PARS[MU2], PARS[EN2], PARS[PX2] / hbar, PARS[EN1_PREV] - PARS[EN1], PARS[EN2_PREV] - PARS[EN2]);
    output.WriteStatus(buf);
}

void BECtwoComponent::call_IM_init() {
    char buf[320];
    snprintf(buf, sizeof buf, "%-7s %-10s %-10s %-15s %-15s %-15s %-10s %-15s %-15s %-15s %-10s %-10s\n", "Iter.",
             "Time", "Norm1", "mu1", "Energy1", "Px1", "Norm2", "mu2", "Energy2", "Px2", "Ediff1", "Ediff2");
    output.CreateStatusFile(buf);
    output.WritePsiInit(psi1.data(), p.Npoints, "1");
    output.WritePsiInit(psi2.data(), p.Npoints, "2");
}

void BECtwoComponent::call_IM_loop_after_step() {
    const int iteration = (int)PARS[ITER];
    if (iteration % itStatMod() == 0) {
        PARS[PX1] = calcPx(0) / (PARS[NORM1] / p.aho1);
        PARS[PX2] = calcPx(1) / (PARS[NORM2] / p.aho1);
        status_line_imag();
    }
    if ((iteration + 1) % p.itmod == 0) {
        write_frames("", "");  // both into psi.wdat, as hamiltonians/BEC_twoComponent.cu:316-317
        PARS[NCYCLES]++;
    }
}

void BECtwoComponent::call_IM_loop_convergence() {
    PARS[PX1] = calcPx(0) / (PARS[NORM1] / p.aho1);
    PARS[PX2] = calcPx(1) / (PARS[NORM2] / p.aho1);
    status_line_imag();
    std::cout << "Convergence reached: dE1 = " << PARS[EN1_PREV] - PARS[EN1] << std::endl;
    std::cout << "                     dE2 = " << PARS[EN2_PREV] - PARS[EN2] << std::endl;
}

void BECtwoComponent::call_IM_end() {
    output.WritePsiFinal(psi1.data(), p.Npoints, "1");
    output.WritePsiFinal(psi2.data(), p.Npoints, "2");
    output.CloseStatusFile();
    output.WriteWtxt_2c(p, (int)PARS[NCYCLES]);
    output.WriteVariable2WTXT("en", PARS[EN1], "code");
    output.WriteVariable2WTXT("en", PARS[EN2], "code");
    output.WriteVariable2WTXT("mu", PARS[MU1], "code");
    output.WriteVariable2WTXT("mu", PARS[MU2], "code");
    output.WriteVariable2WTXT("px", PARS[PX1], "hbar");
    output.WriteVariable2WTXT("px", PARS[PX2], "hbar");
    output.WriteVariable2WTXT("convergence1", PARS[EN1_PREV] - PARS[EN1], "code");
    output.WriteVariable2WTXT("convergence2", PARS[EN2_PREV] - PARS[EN2], "code");
    std::cout << "Average iteration time: " << PARS[AVG_TIME] / PARS[ITER] << std::endl;
    std::cout << "Files saved under prefix: " << p.outpath << std::endl;
}

void BECtwoComponent::status_line_real(double time) {
    char buf[400];
    snprintf(buf, sizeof buf,
             "%-15.5f %-10.4f %-10.1f %-15.12f %-15.12f %-15.12f %-10.1f %-15.12f %-15.12f %-15.12f %-15.12f "
             "%-15.12f %-10.3E %-10.3E\n",
             time, PARS[ITER_TIME], PARS[NORM1], PARS[MU1], PARS[EN1], PARS[PX1], PARS[NORM2], PARS[MU2], PARS[EN2],
             PARS[PX2], PARS[AUX1_1], PARS[AUX1_2], PARS[EN1] - PARS[EN1_0], PARS[EN2] - PARS[EN2_0]);
    output.WriteStatus(buf);
}

// hamiltonians/BEC_twoComponent.cu:383-416
void BECtwoComponent::call_RE_init() {
    char buf[400];
    snprintf(buf, sizeof buf, "%-15s %-10s %-10s %-15s %-15s %-15s %-10s %-15s %-15s  %-15s %-15s %-15s %-10s %-10s\n",
             "Time", "ItTime", "Norm1", "mu1", "Energy1", "Px1", "Norm2", "mu2", "Energy2", "Px2", "<cos_1>",
             "<cos_2>", "Ediff1", "Ediff2");
    output.CreateStatusFile(buf);
    output.WriteWtxt_2c(p, 0);
    output.WritePsiInit(psi1.data(), p.Npoints, "1");
    output.WritePsiInit(psi2.data(), p.Npoints, "2");
    PARS[NORM1] = p.npart1;
    PARS[NORM2] = p.npart2;
    double o[6];
    chk(gpe_observables(h, 0.0, o), "gpe_observables");
    PARS[MU1_0] = o[1] / PARS[NORM1];
    PARS[EN1_0] = o[2] / PARS[NORM1];
    PARS[MU2_0] = o[4] / PARS[NORM2];
    PARS[EN2_0] = o[5] / PARS[NORM2];
    PARS[NORM1] = o[0];
    PARS[NORM2] = o[3];
    double c1 = 0.0, c2 = 0.0;
    chk(gpe_average_cos(h, 0, &c1), "gpe_average_cos");
    chk(gpe_average_cos(h, 1, &c2), "gpe_average_cos");
    PARS[AUX1_1] = c1 / PARS[NORM1];
    PARS[AUX1_2] = c2 / PARS[NORM2];
    PARS[PX1] = calcPx(0) / ((PARS[NORM1] * hbar) / p.aho1);
    PARS[PX2] = calcPx(1) / ((PARS[NORM2] * hbar) / p.aho1);
    status_line_real(0.0);
}

// hamiltonians/BEC_twoComponent.cu:425-466 (status observables with H of the
// current psi; the reference pairs psi with stale hpsi buffers there)
void BECtwoComponent::call_RE_loop_after_step() {
    if (((int)PARS[ITER]) % itStatMod() == 0) {
        double o[6];
        chk(gpe_observables(h, 0.0, o), "gpe_observables");
        PARS[NORM1] = o[0];
        PARS[NORM2] = o[3];
        PARS[MU1] = o[1] / PARS[NORM1];
        PARS[EN1] = o[2] / PARS[NORM1];
        PARS[MU2] = o[4] / PARS[NORM2];
        PARS[EN2] = o[5] / PARS[NORM2];
        double c1 = 0.0, c2 = 0.0;
        chk(gpe_average_cos(h, 0, &c1), "gpe_average_cos");
        chk(gpe_average_cos(h, 1, &c2), "gpe_average_cos");
        PARS[AUX1_1] = c1 / PARS[NORM1];
        PARS[AUX1_2] = c2 / PARS[NORM2];
        PARS[PX1] = calcPx(0) / ((PARS[NORM1] * hbar) / p.aho1);
        PARS[PX2] = calcPx(1) / ((PARS[NORM2] * hbar) / p.aho1);
        status_line_real(p.time0 + PARS[ITER] * p.dt);
    }
    if (((int)PARS[ITER] + 1) % p.itmod == 0) {
        write_frames("1", "2");
        PARS[NCYCLES]++;
    }
}

void BECtwoComponent::call_RE_end() {
    output.WritePsiFinal(psi1.data(), p.Npoints, "1");
    output.WritePsiFinal(psi2.data(), p.Npoints, "2");
    output.CloseStatusFile();
    output.WriteWtxt_2c(p, (int)PARS[NCYCLES]);
    output.WriteVariable2WTXT("en10", PARS[EN1_0], "code");
    output.WriteVariable2WTXT("en20", PARS[EN2_0], "code");
    output.WriteVariable2WTXT("mu10", PARS[MU1_0], "code");
    output.WriteVariable2WTXT("mu20", PARS[MU2_0], "code");
    output.WriteVariable2WTXT("en1", PARS[EN1], "code");
    output.WriteVariable2WTXT("en1", PARS[EN2], "code");
    output.WriteVariable2WTXT("mu1", PARS[MU1_0], "code");
    output.WriteVariable2WTXT("mu2", PARS[MU2_0], "code");
    output.WriteVariable2WTXT("px1", PARS[PX1], "hbar");
    output.WriteVariable2WTXT("px2", PARS[PX2], "hbar");
    std::cout << "Average iteration time: " << PARS[AVG_TIME] / PARS[ITER] << std::endl;
    std::cout << "Files saved under prefix: " << p.outpath << std::endl;
}

// ==== main.cu:20-82 ==========================================================================
int run_input_file(const std::string& file) {
    try {
        InputVariables reader(file);
        if (!reader.getBool("t2component")) {
            std::cout << "# Single component mode." << std::endl;
            Params params(reader);
            const std::string hm = params.getString("hamiltonian");
            if (hm == "bec") {
                std::cout << "# BEC hamiltonian" << std::endl;
                BEConeComponent bec(params);
            } else if (hm == "template") {
                SingleTemplate t(params);
            } else if (hm == "dbec") {
                std::cout << "# dipolar BEC hamiltonian" << std::endl;
                BEConeComponent bec(params, true, GPE_HAM_DIPOLAR);
            } else {
                std::cerr << "No hamiltonian available for: " << hm << std::endl;
                return 1;
            }
        } else {
            std::cout << "# Two component mode." << std::endl;
            Params2 params2(reader);
            const std::string hm = params2.getString("hamiltonian");
            if (hm == "2bec") {
                std::cout << "# 2BEC hamiltonian" << std::endl;
                BECtwoComponent bec(params2);
            } else {
                std::cerr << "No hamiltonian available for: " << hm << std::endl;
                return 2;
            }
        }
    } catch (const HostError& e) {
        std::cerr << e.what() << std::endl;
        return 3;
    }
    return 0;
}

}  // namespace gpe
