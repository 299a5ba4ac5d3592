"""Host-side logic that needs no GPU: configuration round trips, scheme dispatch,
parameter packing and the Runge-Kutta tableaux."""
import pytest

import warpsph_b200 as ws
from warpsph_b200 import configurations as cf
from warpsph_b200.integrators import _TABLEAUX


def test_build_scheme_tuple_and_errors():
    t = ws.buildScheme("crkSPH")
    assert len(t) == 7
    System, State, Config, Update, step, to_dict, from_dict = t
    assert System is ws.CompSPHSystem and State is ws.CompSPHState and Config is ws.CRKSPHConfig
    assert step is ws.crkSPH_step
    assert ws.buildScheme(ws.CompressibleSPHScheme.CRKSPH)[4] is ws.crkSPH_step
    with pytest.raises(ValueError):
        ws.buildScheme("notAScheme")


def test_config_round_trips():
    c = ws.CRKSPHConfig()
    c.viscositySwitchParams.scheme = ws.ViscositySwitch.CullenDehnen2010
    c.crkViscosityParams.eta_crit = 0.25
    d = ws.crkSPHConfigToDict(c)
    c2 = ws.dictToCRKSPHConfig(d)
    assert c2 == c
    s, _ = ws.buildConfig(dim=2, domain=ws.buildDomainDescription(1.0, 2, True), kernel=ws.KernelFunctions.Wendland4)
    s2 = ws.dictToConfig(ws.configurationToDict(s))
    assert s2.kernel == s.kernel and s2.verletScale == s.verletScale and s2.domain.host() == s.domain.host()


def test_defaults_follow_reference():
    s, integ = ws.buildConfig()
    assert s.integrationScheme == ws.IntegrationSchemeType.rungeKutta2
    assert abs(s.verletScale - 2 ** 0.5) < 1e-12
    c = ws.CRKSPHConfig()
    assert c.energyScheme == ws.EnergyScheme.CRK and c.compatibleEnergy
    assert c.diffusionParams.C_l == 1 and c.diffusionParams.C_q == 1
    assert c.crkViscosityParams.eta_crit == 0.3333333 and c.crkViscosityParams.eta_fold == 0.2
    assert c.viscositySwitchParams.limitXi is True and c.viscositySwitchParams.alpha_max == 2.0
    assert abs(ws.n_h_to_nH(4, 2) - 16 * 3.141592653589793) < 1e-9


def test_make_params_packs_config():
    s, _ = ws.buildConfig(dim=3, domain=ws.buildDomainDescription(2.0, 3, False), kernel=ws.KernelFunctions.Wendland2)
    c = ws.CRKSPHConfig()
    c.gamma = 5 / 3
    p = cf.make_params(s, c)
    assert p.dim == 3 and p.kernel == 1 and list(p.domain_min) == [-1.0] * 3 and list(p.periodic) == [0, 0, 0]
    assert abs(p.gamma - 5 / 3) < 1e-15 and p.energy_scheme == 5 and p.enable_crk_limiter == 1


@pytest.mark.parametrize("scheme", list(_TABLEAUX))
def test_tableaux_are_consistent(scheme):
    a, b, c = _TABLEAUX[scheme]
    assert abs(sum(b) - 1) < 1e-15
    for s, row in enumerate(a):
        assert abs(sum(row) - c[s]) < 1e-15
