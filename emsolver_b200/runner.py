"""Set up a TlmSolver from a synthetic Workload (emsolver_b200.workloads)."""
from __future__ import annotations

from .solver import MatProps, TlmConfig, TlmSolver, VoxelGridSpec


def build_solver(w, device: int = 0, storage: int | None = None, steps_per_launch: int = 0,
                 variant: str | None = None, pulse_scale: float = 0.0, kernel_variant: int = 0,
                 rounding: int = 0, general_tiles: bool = False, no_staging: bool = False,
                 stage_wait_us: int = 0, near_field: int | None = None) -> TlmSolver:
    """Create, set up and populate a solver exactly as the reference would be:
    setup, ports (in order), plane wave, probes at cell centres, port DFT."""
    s = TlmSolver(device, variant)
    grid = VoxelGridSpec(w.nx, w.ny, w.nz, tuple(w.origin), w.dl)
    cfg = TlmConfig(f0=w.f0, waveform=w.waveform, totalSteps=w.steps, settleSteps=w.meta.get("settle_steps", 0),
                    huyOffset=w.meta.get("huy_offset", 0), recordEvery=w.meta.get("record_every", 0),
                    surfaceMonitors=bool(w.meta.get("surface_monitors", False)),
                    boundaryRho=w.rho, storage=w.storage if storage is None else storage,
                    stepsPerLaunch=steps_per_launch, pulseScale=pulse_scale,
                    kernelVariant=kernel_variant, rounding=rounding, generalTiles=general_tiles,
                    noStaging=no_staging, stageWaitUs=stage_wait_us,
                    nearField=w.meta.get("near_field", 0) if near_field is None else near_field)
    s.setup(grid, w.mat, [MatProps(e, g) for e, g in w.table], cfg)
    if w.waveform == 3 and w.sv is not None:
        s.setSourceTable(w.sv)
    for cells, pol, amp in w.ports:
        s.addPort(cells, pol, amp)
    if "plane_wave" in w.meta:
        s.addPlaneWave(*w.meta["plane_wave"])
    for (i, j, k) in w.probes_cell:
        s.addProbe(w.cell_center(i, j, k))
    if w.dft_freqs is not None:
        s.setPortDft(w.dft_freqs)
    if "field_plane" in w.meta:
        s.setFieldPlane(*w.meta["field_plane"])
    return s


def records(s, w, f64: bool = False):
    """Records in the oracle's naming (see oracle/drive.py)."""
    out = {}
    for p in range(len(w.ports)):
        port = s.port(p, f64=f64)
        out[f"port{p}_v"] = port.vRec
        out[f"port{p}_i"] = port.iRec
    for q in range(len(w.probes_cell)):
        pr = s.probe(q, f64=f64)
        out[f"probe{q}_ex"] = pr.ex
        out[f"probe{q}_ey"] = pr.ey
        out[f"probe{q}_ez"] = pr.ez
    st, ev = s.getEnergyHistory(f64=True)
    out["energy_steps"] = st
    out["energy"] = ev
    return out
