// tlm_b200.hpp -- C++ mirror of smilima/EMSolver's TlmSolver (TlmSolver.h:202-264)
// over the C ABI in tlm_b200.h. Header-only; link libtlm_b200.so.
//
// Same method names, argument meaning and result types as the reference, so a
// caller such as TMainForm::startSimulation (MainUnit.cpp:872-991) or
// BuildDipoleSim (SelfTest.cpp:98-178) can switch by changing the type:
//   setup(grid, materials, matTable, cfg)      TlmSolver.cpp:259-304
//   addPort(cells, polAxis, amp) -> index       TlmSolver.cpp:362-374
//   addPlaneWave(propAxis, planeIndex, polAxis, amp)
//   addProbe(worldPos) -> index or -1           TlmSolver.cpp:377-391
//   run() / requestStop() / currentStep() / currentEnergy() / isRunning()
//   probe(i) -> FieldProbe, ports() -> TlmPort records, getEnergyHistory()
// Differences: errors throw tlmb200::Error (the reference has no error path
// for these calls), and records are fetched from the device on request.
#ifndef TLM_B200_HPP
#define TLM_B200_HPP

#include "tlm_b200.h"

#include <cstddef>
#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

namespace tlmb200 {

class Error : public std::runtime_error
{
public:
    Error(tlm_status s, const std::string &m) : std::runtime_error(m), status(s) {}
    tlm_status status;
};

struct Vec3
{
    float x = 0, y = 0, z = 0;
};

struct VoxelGridSpec  // Geometry.h:85-113
{
    int nx = 0, ny = 0, nz = 0;
    Vec3 origin;
    float dl = 1e-3f;
    size_t cellIndex(int i, int j, int k) const { return ((size_t)k * ny + j) * nx + i; }
};

struct MatProps  // TlmSolver.h:61-65
{
    float epsr = 1.0f;
    float sigma = 0.0f;
};

enum class WaveformType { CwRamped = 0, GaussianSine = 1, GaussianPulse = 2, Table = 3 };
enum class Storage { F32 = TLM_STORE_F32, BF16 = TLM_STORE_BF16, F16 = TLM_STORE_F16, F64 = TLM_STORE_F64 };

struct TlmConfig  // TlmSolver.h:113-123 (+ storage, pulse scale, steps per launch)
{
    float f0 = 1e9f;
    WaveformType waveform = WaveformType::CwRamped;
    int totalSteps = 2000;
    int settleSteps = 600;
    float boundaryRho = 0.0f;
    int huyOffset = 0;
    bool useGpu = true;
    int recordEvery = 0;
    Storage storage = Storage::F32;
    float pulseScale = 0.0f;
    int stepsPerLaunch = 0;
    int kernelVariant = 0;
    int rounding = 0;  // BF16/F16 storage: 0 nearest, 1 stochastic
};

struct TlmPort  // TlmSolver.h:81-87
{
    std::vector<size_t> cells;
    int polAxis = 2;
    float amp = 1.0f;
    std::vector<float> vRec, iRec;
};

struct FieldProbe  // TlmSolver.h:136-141
{
    size_t cell = 0;
    Vec3 pos;
    std::vector<float> ex, ey, ez;
};

class TlmSolver
{
public:
    explicit TlmSolver(int device = 0)
    {
        check(tlm_create(&h_, device), nullptr);
    }
    ~TlmSolver() { tlm_destroy(h_); }
    TlmSolver(const TlmSolver &) = delete;
    TlmSolver &operator=(const TlmSolver &) = delete;

    void setup(const VoxelGridSpec &grid, std::vector<uint8_t> materials,
               std::vector<MatProps> matTable, const TlmConfig &cfg)
    {
        tlm_grid g{ grid.nx, grid.ny, grid.nz, { grid.origin.x, grid.origin.y, grid.origin.z },
                    grid.dl };
        std::vector<tlm_matprops> tab(matTable.size());
        for (size_t t = 0; t < matTable.size(); ++t) tab[t] = { matTable[t].epsr, matTable[t].sigma };
        tlm_config c;
        tlm_config_default(&c);
        c.f0 = cfg.f0;
        c.waveform = (int)cfg.waveform;
        c.total_steps = cfg.totalSteps;
        c.settle_steps = cfg.settleSteps;
        c.boundary_rho = cfg.boundaryRho;
        c.huy_offset = cfg.huyOffset;
        c.use_gpu = 1;
        c.record_every = cfg.recordEvery;
        c.storage = (int)cfg.storage;
        c.pulse_scale = cfg.pulseScale;
        c.steps_per_launch = cfg.stepsPerLaunch;
        c.kernel_variant = cfg.kernelVariant;
        c.rounding = cfg.rounding;
        check(tlm_setup(h_, &g, materials.data(), materials.size(), tab.data(), (int)tab.size(), &c));
        grid_ = grid;
        cfg_ = cfg;
        meta_.clear();
        probePos_.clear();
    }

    int addPort(const std::vector<size_t> &cells, int polAxis, float amp)
    {
        std::vector<uint64_t> c(cells.begin(), cells.end());
        int idx = -1;
        check(tlm_add_port(h_, c.data(), (int)c.size(), polAxis, amp, &idx));
        meta_.push_back({ polAxis, amp });
        return idx;
    }
    void addPlaneWave(int propAxis, int planeIndex, int polAxis, float amp)
    {
        check(tlm_add_plane_wave(h_, propAxis, planeIndex, polAxis, amp));
    }
    int addProbe(const Vec3 &worldPos)
    {
        int idx = -1;
        check(tlm_add_probe(h_, worldPos.x, worldPos.y, worldPos.z, &idx));
        if (idx >= 0) probePos_.push_back(worldPos);
        return idx;
    }
    void setSourceTable(const std::vector<float> &sv)
    {
        check(tlm_set_source_table(h_, sv.data(), (int)sv.size()));
    }
    void setPortDft(const std::vector<double> &freqs)
    {
        check(tlm_set_port_dft(h_, freqs.data(), (int)freqs.size()));
    }

    // Blocking, like the reference's run(); false if requestStop ended it.
    bool run()
    {
        tlm_status s = tlm_run(h_);
        if (s == TLM_ESTOPPED) return false;
        check(s);
        return true;
    }
    void step(int n) { check(tlm_step(h_, n)); }
    void requestStop() { tlm_request_stop(h_); }
    bool isRunning() const { return tlm_is_running(h_) != 0; }
    bool isFinished() const { return tlm_is_finished(h_) != 0; }
    int currentStep() const { return tlm_current_step(h_); }
    int totalSteps() const { return tlm_total_steps(h_); }
    float currentEnergy() const { return tlm_current_energy(h_); }
    bool ranOnGpu() const { return true; }
    const VoxelGridSpec &grid() const { return grid_; }
    const TlmConfig &cfg() const { return cfg_; }
    float timestep() const
    {
        float dt = 0.0f;
        tlm_timestep(h_, &dt);
        return dt;
    }

    int probeCount() const { return tlm_probe_count(h_); }
    FieldProbe probe(int idx) const
    {
        FieldProbe p;
        int n = 0;
        check(tlm_get_probe(h_, idx, nullptr, nullptr, nullptr, 0, &n));
        p.ex.resize(n);
        p.ey.resize(n);
        p.ez.resize(n);
        check(tlm_get_probe(h_, idx, p.ex.data(), p.ey.data(), p.ez.data(), n, &n));
        uint64_t cell = 0;
        check(tlm_get_probe_cell(h_, idx, &cell));
        p.cell = (size_t)cell;
        if (idx >= 0 && idx < (int)probePos_.size()) p.pos = probePos_[idx];
        return p;
    }

    std::vector<TlmPort> ports() const
    {
        std::vector<TlmPort> out(tlm_port_count(h_));
        for (int i = 0; i < (int)out.size(); ++i)
        {
            int n = 0, nc = 0;
            check(tlm_get_port(h_, i, nullptr, nullptr, 0, &n));
            out[i].vRec.resize(n);
            out[i].iRec.resize(n);
            check(tlm_get_port(h_, i, out[i].vRec.data(), out[i].iRec.data(), n, &n));
            check(tlm_get_port_cells(h_, i, nullptr, 0, &nc));
            std::vector<uint64_t> c(nc);
            check(tlm_get_port_cells(h_, i, c.data(), nc, &nc));
            out[i].cells.assign(c.begin(), c.end());
            if (i < (int)meta_.size())
            {
                out[i].polAxis = meta_[i].first;
                out[i].amp = meta_[i].second;
            }
        }
        return out;
    }

    void getEnergyHistory(std::vector<int> &steps, std::vector<float> &vals) const
    {
        int n = 0;
        check(tlm_get_energy_history(h_, nullptr, nullptr, nullptr, 0, &n));
        steps.resize(n);
        vals.resize(n);
        check(tlm_get_energy_history(h_, steps.data(), vals.data(), nullptr, n, &n));
    }

    static float ScatterUnitarityError(int device = 0)
    {
        float e = 0.0f;
        check(tlm_scatter_unitarity_error(device, &e), nullptr);
        return e;
    }
    static float DielScatterUnitarityError(float epsr, int device = 0)
    {
        float e = 0.0f;
        check(tlm_stub_unitarity_error(device, epsr, &e), nullptr);
        return e;
    }

    tlm_handle handle() const { return h_; }

private:
    void check(tlm_status s) const { check(s, h_); }
    static void check(tlm_status s, tlm_handle h)
    {
        if (s != TLM_OK) throw Error(s, tlm_last_error(h));
    }

    tlm_handle h_ = nullptr;
    VoxelGridSpec grid_;
    TlmConfig cfg_;
    std::vector<std::pair<int, float>> meta_;
    std::vector<Vec3> probePos_;
};

} // namespace tlmb200

#endif // TLM_B200_HPP
