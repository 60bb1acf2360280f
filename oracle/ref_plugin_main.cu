// ref_plugin_main.cu -- test plugins + main for the reference's own CUDA build
// (TEST INFRASTRUCTURE; built only into oracle/_ref/gpe_ref_trace by
// oracle/ref.mk, run only on a GPU host to make golden fixtures and to time
// the reference).
//
// Why: the shipped "bec" plugin only sets d_h_params[0] = a
// (hamiltonians/BEC_oneComponent.cu:14) and d_quench_as then returns
// prms[2] = 0 for every t (hamiltonians/BEC_oneComponent.cu:167-178), so the
// stock binary always runs with g = 0.  These plugins follow the reference's
// documented plugin contract (hamiltonians/BEC_oneComponent.hpp:8-22): they
// derive from its solver classes, build Psi/Vext with its classes, fill
// d_h_params from the input file and launch the reference's own Hamiltonian
// kernels.  Hooks write a full-precision trace of the PARS the reference
// computes, plus psi_final.wdat through its Output class.
//
// Extra input keys (all optional):
//   quench_f0 quench_f1 quench_f2  -> prms[0..2] = a * f   (default 1 1 1)
//   quench_t1 quench_t2 quench_t3  -> prms[3..5]           (default 0 0 0)
//   trace_every                    -> trace stride of real-time steps (default itStatMod)
#include "hamiltonians/BEC_oneComponent.hpp"
#include "hamiltonians/BEC_twoComponent.hpp"
#include "hamiltonians/single_template.hpp"
#include "input_variables.hpp"
#include "params.hpp"
#include "params2.hpp"

#include <chrono>
#include <cstdio>
#include <cstring>
#include <string>

// Wall time of the reference's own evolution loop (runRealTimeEvol /
// runImagTimeEvol), device-synchronised on both sides, printed to stderr as
// "ref_loop_seconds <s>" for oracle/time_ref_build.py: process start-up,
// cuFFT plan creation and the initial-state set-up stay outside it.
template <typename F>
static void timed_loop(F&& run) {
    cudaDeviceSynchronize();
    const auto t0 = std::chrono::steady_clock::now();
    run();
    cudaDeviceSynchronize();
    const auto t1 = std::chrono::steady_clock::now();
    std::fprintf(stderr, "ref_loop_seconds %.9f\n", std::chrono::duration<double>(t1 - t0).count());
}

namespace {
double opt_double(const ParamsBase& p, const char* key, double dflt) {
    return (p.getIV().getVariable(key) != "None") ? p.getDouble(key) : dflt;
}
int opt_int(const ParamsBase& p, const char* key, int dflt) {
    return (p.getIV().getVariable(key) != "None") ? p.getInt(key) : dflt;
}
}  // namespace

class TracePlugin1 : public OneComponentGPSolver {
public:
    Params p;
    int kind;  // 0: BEC kernels, 1: single_template kernels
    FILE* trace = nullptr;
    int trace_every = 1;

    TracePlugin1(Params& par, int kind_) : OneComponentGPSolver(par), kind(kind_) {
        this->p = par;
        {
            Psi* ps = new Psi(p, std::string(""));
            if (p.getBool("tpi_vortex")) ps->imprintVortexTube(p, p.getDouble("api_prc"));
            std::memcpy(this->psi, ps->getPsi(), p.Npoints * sizeof(complex));
            delete ps;
        }
        {
            Vext* v = new Vext(p, std::string(""));
            if (p.getBool("tvseed")) v->addProtocolPotential(p, 0);
            std::memcpy(this->vext, v->getVext(), p.Npoints * sizeof(complex));
            delete v;
        }
        double hp[NO_HAMIL_PARAMS] = {0};
        hp[0] = p.a * opt_double(p, "quench_f0", 1.0);
        hp[1] = p.a * opt_double(p, "quench_f1", 1.0);
        hp[2] = p.a * opt_double(p, "quench_f2", 1.0);
        hp[3] = opt_double(p, "quench_t1", 0.0);
        hp[4] = opt_double(p, "quench_t2", 0.0);
        hp[5] = opt_double(p, "quench_t3", 0.0);
        CCE(cudaMemcpy(this->d_h_params, hp, NO_HAMIL_PARAMS * sizeof(double), cudaMemcpyHostToDevice), "h_params");
        trace_every = opt_int(p, "trace_every", p.getInt("itStatMod"));
        trace = fopen((p.outpath + "trace.txt").c_str(), "w");
        output.WritePsiInit(this->psi, p.Npoints);
        output.WriteVext(this->vext, p.Npoints);
        timed_loop([&] {
            if (p.getBool("treal")) runRealTimeEvol();
            else runImagTimeEvol();
        });
        fclose(trace);
    }

    void alg_calcHpsi() override {
        this->alg_Laplace(this->d_psi, this->d_hpsi);
        if (kind == 0)
            BECHamiltonian<<<gridSize, noThreads, 0, stream>>>(PARS[T], this->d_psi, this->d_hpsi, this->d_vext,
                                                                this->d_hpsi_en, this->d_hpsi, p.Npoints, this->d_h_params);
        else
            SingleTemplate_template<<<gridSize, noThreads, 0, stream>>>(this->d_psi, this->d_hpsi, this->d_vext,
                                                                         this->d_hpsi_en, this->d_hpsi, p.Npoints, this->d_h_params);
    }
    void alg_calcHpsiMU() override {
        this->alg_Laplace(this->d_psi, this->d_hpsi);
        if (kind == 0)
            BECHamiltonianMU<<<gridSize, noThreads, 0, stream>>>(PARS[T], this->d_psi, this->d_hpsi, this->d_vext,
                                                                  this->d_hpsi, p.Npoints, this->d_h_params);
        else
            SingleTemplateMU_template<<<gridSize, noThreads, 0, stream>>>(this->d_psi, this->d_hpsi, this->d_vext,
                                                                           this->d_hpsi, p.Npoints, this->d_h_params);
    }

    void line(const char* tag) {
        fprintf(trace, "%s %d %.17g %.17g %.17g %.17g\n", tag, (int)PARS[ITER], PARS[NORM], PARS[MU], PARS[EN], PARS[EN_PREV]);
    }
    void call_IM_init() override {}
    void call_IM_loop_before_step() override {}
    void call_IM_loop_after_step() override { line("im"); }
    void call_IM_loop_convergence() override { line("conv"); }
    void call_IM_end() override {
        output.WritePsiFinal(this->psi, p.Npoints);
        fprintf(trace, "end %d\n", (int)PARS[ITER]);
    }
    void call_RE_init() override {}
    void call_RE_loop_before_step() override {}
    // Same reductions as hamiltonians/BEC_oneComponent.cu:347-348.
    void call_RE_loop_after_step() override {
        if (((int)PARS[ITER]) % trace_every == 0) {
            this->alg_calcNorm(&PARS[NORM], this->d_psi);
            this->alg_calc2Observables(PARS[NORM], &PARS[MU], &PARS[EN], this->d_psi, this->d_hpsi, this->d_hpsi_en);
            line("re");
        }
    }
    void call_RE_end() override {
        cudaStreamSynchronize(streamData);
        output.WritePsiFinal(this->psi, p.Npoints);
        fprintf(trace, "end %d\n", (int)PARS[ITER]);
    }
};

class TracePlugin2 : public TwoComponentGPSolver {
public:
    Params2 p;
    FILE* trace = nullptr;
    int trace_every = 1;

    explicit TracePlugin2(Params2& par) : TwoComponentGPSolver(par) {
        this->p = par;
        for (int c = 1; c <= 2; ++c) {
            Psi* ps = new Psi(p, c);
            if (p.getBool("tpi_vortex")) ps->imprintVortexTube(p, p.getDouble("api_prc"));
            std::memcpy(c == 1 ? this->psi1 : this->psi2, ps->getPsi(), p.Npoints * sizeof(complex));
            delete ps;
            Vext* v = new Vext(p, c);
            if (p.getBool("tvseed")) v->addWeightedProtocolPotential(p, c);
            std::memcpy(c == 1 ? this->vext1 : this->vext2, v->getVext(), p.Npoints * sizeof(complex));
            delete v;
        }
        double hp[NO_HAMIL_PARAMS] = {0};
        hp[0] = p.a11;
        hp[1] = p.a22;
        hp[2] = p.a12;
        CCE(cudaMemcpy(this->d_h_params, hp, NO_HAMIL_PARAMS * sizeof(double), cudaMemcpyHostToDevice), "h_params");
        trace_every = opt_int(p, "trace_every", p.getInt("itStatMod"));
        trace = fopen((p.outpath + "trace.txt").c_str(), "w");
        output.WritePsiInit(this->psi1, p.Npoints, "1");
        output.WritePsiInit(this->psi2, p.Npoints, "2");
        output.WriteVext(this->vext1, p.Npoints, "1");
        output.WriteVext(this->vext2, p.Npoints, "2");
        timed_loop([&] {
            if (p.getBool("treal")) runRealTimeEvol();
            else runImagTimeEvol();
        });
        fclose(trace);
    }

    void alg_calcHpsi() override {
        this->alg_Laplace(this->d_psi, this->d_hpsi);
        this->alg_Laplace(this->d_psi2, this->d_hpsi2);
        BECHamiltonian_2<<<gridSize, noThreads, 0, stream>>>(this->d_psi, this->d_psi2, this->d_hpsi, this->d_hpsi2,
                                                              this->d_vext, this->d_vext2, this->d_hpsi_en, this->d_hpsi2_en,
                                                              p.Npoints, this->d_h_params);
    }
    void alg_calcHpsiMU() override {
        this->alg_Laplace(this->d_psi, this->d_hpsi);
        this->alg_Laplace(this->d_psi2, this->d_hpsi2);
        BECHamiltonianMU_2<<<gridSize, noThreads, 0, stream>>>(this->d_psi, this->d_psi2, this->d_hpsi, this->d_hpsi2,
                                                                this->d_vext, this->d_vext2, p.Npoints, this->d_h_params);
    }
    void line(const char* tag) {
        fprintf(trace, "%s %d %.17g %.17g %.17g %.17g %.17g %.17g %.17g %.17g\n", tag, (int)PARS[ITER],
                PARS[NORM1], PARS[MU1], PARS[EN1], PARS[EN1_PREV], PARS[NORM2], PARS[MU2], PARS[EN2], PARS[EN2_PREV]);
    }
    void call_IM_init() override {}
    void call_IM_loop_before_step() override {}
    void call_IM_loop_after_step() override { line("im"); }
    void call_IM_loop_convergence() override { line("conv"); }
    void call_IM_end() override {
        output.WritePsiFinal(this->psi1, p.Npoints, "1");
        output.WritePsiFinal(this->psi2, p.Npoints, "2");
        fprintf(trace, "end %d\n", (int)PARS[ITER]);
    }
    void call_RE_init() override {}
    void call_RE_loop_before_step() override {}
    void call_RE_loop_after_step() override {}
    void call_RE_end() override {
        output.WritePsiFinal(this->psi1, p.Npoints, "1");
        output.WritePsiFinal(this->psi2, p.Npoints, "2");
        fprintf(trace, "end %d\n", (int)PARS[ITER]);
    }
};

// main.cu:20-82 dispatch with the test plugins.  Plugins are never deleted:
// TwoComponentGPSolver's destructor free()s host axes that BaseHamiltonian
// allocated with cudaMallocHost (hpp/twoComponentGPSolver.hpp:50-61,
// src/baseHamiltonian.cu:27-29,57-59).
int main(int argc, const char* argv[]) {
    if (argc != 2) {
        std::cerr << "Usage: " << argv[0] << " <filename>" << std::endl;
        return 1;
    }
    InputVariables reader{std::string(argv[1])};
    if (!reader.getBool("t2component")) {
        Params params(reader);
        std::string h = params.getString("hamiltonian");
        if (h == "bec") new TracePlugin1(params, 0);
        else if (h == "template") new TracePlugin1(params, 1);
        else { std::cerr << "No hamiltonian available for: " << h << std::endl; return 1; }
    } else {
        Params2 params2(reader);
        std::string h = params2.getString("hamiltonian");
        if (h == "2bec") new TracePlugin2(params2);
        else { std::cerr << "No hamiltonian available for: " << h << std::endl; return 2; }
    }
    cudaDeviceSynchronize();
    return 0;
}
