"""A resumed run equals the uninterrupted run bit for bit: a CRKSPH Sedov system is
exported after two RK2 steps (src/warpSPH/io.py layout, with the stages), imported in
place of the live system, and both continue for three more steps on the GPU."""
import pytest
import torch

import warpsph_b200 as ws
from warpsph_b200 import io

pytestmark = pytest.mark.gpu

FIELDS = ("positions", "velocities", "internalEnergies", "densities", "supports", "pressures", "soundspeeds", "alphas", "alpha0s",
          "divergence", "entropies")


def test_resume_from_export_is_bit_identical(cuda, tmp_path):
    cfg, integ = ws.buildConfig(dim=2, domain=ws.buildDomainDescription(1.0, 2, True, cuda), kernel=ws.KernelFunctions.Wendland4,
                                targetNeighbors=32, device=cuda)
    System, State, Config, Update, step, *_ = ws.buildScheme("crkSPH")
    sch = Config()
    sch.gamma = 5 / 3
    sch.viscositySwitchParams.scheme = ws.ViscositySwitch.CullenDehnen2010
    system = ws.buildSedov(System, State, cfg, nx=48, dim=2, domainExtent=1.0, gamma=5 / 3, kernel=ws.KernelFunctions.Wendland4,
                           targetNeighbors=32, device=cuda)
    dt = 1e-4
    res = None
    for _ in range(2):
        res = integ.function(state=system, f=step, dt=dt, config=cfg, compParams=sch)
        system = res.state
    path = io.exportSimulationSystem(str(tmp_path), "resume", ws.CompressibleSPHScheme.CRKSPH, system, stages=res.stages,
                                     extraData={"frame_num": 2})
    live = system
    for _ in range(3):
        live = integ.function(state=live, f=step, dt=dt, config=cfg, compParams=sch).state
    resumed, stages, scheme, extra = io.importSimulationSystem(path, cuda, torch.float32)
    resumed.domain = live.domain
    assert scheme == ws.CompressibleSPHScheme.CRKSPH and extra["frame_num"] == 2 and len(stages) == 2
    for _ in range(3):
        resumed = integ.function(state=resumed, f=step, dt=dt, config=cfg, compParams=sch).state
    torch.cuda.synchronize()
    for name in FIELDS:
        a, b = getattr(live.state, name), getattr(resumed.state, name)
        assert torch.equal(a, b), f"{name}: max |diff| {(a - b).abs().max().item():.3g}"
    assert resumed.t == pytest.approx(live.t)
