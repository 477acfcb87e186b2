// tlm_cpp_client.cpp -- a C++ caller of the library through include/tlm_b200.hpp,
// written the way the reference's own callers drive TlmSolver
// (SelfTest.cpp:98-178: setup, addPort, run on a thread while polling
// currentStep/currentEnergy, then read the records).
//
// Usage: tlm_cpp_client <out.bin>
// Runs 64^3 free space, rho = 0, GaussianPulse of width 20 steps on the
// centre node's Ez links, probe at (48,32,32), 500 steps; writes the probe's
// Ez series (500 floats) followed by the port V and I series.
#include "tlm_b200.hpp"

#include <cstdio>
#include <thread>

int main(int argc, char **argv)
{
    if (argc < 2)
    {
        std::fprintf(stderr, "usage: %s out.bin\n", argv[0]);
        return 2;
    }
    try
    {
        const int n = 64;
        tlmb200::VoxelGridSpec g;
        g.nx = g.ny = g.nz = n;
        g.dl = 1e-3f;
        tlmb200::TlmConfig cfg;
        cfg.f0 = 299792458.0f / (20.0f * g.dl);
        cfg.waveform = tlmb200::WaveformType::GaussianPulse;
        cfg.totalSteps = 500;
        cfg.boundaryRho = 0.0f;
        tlmb200::TlmSolver s(0);
        s.setup(g, std::vector<uint8_t>((size_t)n * n * n, 0), {}, cfg);
        s.addPort({ g.cellIndex(32, 32, 32) }, 2, 1.0f);
        tlmb200::Vec3 p{ (48 + 0.5f) * g.dl, (32 + 0.5f) * g.dl, (32 + 0.5f) * g.dl };
        if (s.addProbe(p) != 0) return 3;
        bool ok = false;
        std::thread th([&] { ok = s.run(); });
        float peakE = 0.0f;
        while (!s.isFinished()) peakE = std::max(peakE, s.currentEnergy());
        th.join();
        if (!ok || s.currentStep() != 500) return 4;
        tlmb200::FieldProbe pr = s.probe(0);
        std::vector<tlmb200::TlmPort> ports = s.ports();
        FILE *f = std::fopen(argv[1], "wb");
        if (!f) return 5;
        std::fwrite(pr.ez.data(), sizeof(float), pr.ez.size(), f);
        std::fwrite(ports[0].vRec.data(), sizeof(float), ports[0].vRec.size(), f);
        std::fwrite(ports[0].iRec.data(), sizeof(float), ports[0].iRec.size(), f);
        std::fclose(f);
        std::printf("ok: %zu samples, unitarity %.3g\n", pr.ez.size(),
                    tlmb200::TlmSolver::ScatterUnitarityError());
        return 0;
    }
    catch (const tlmb200::Error &e)
    {
        std::fprintf(stderr, "tlm error %d: %s\n", (int)e.status, e.what());
        return 1;
    }
}
