"""Host-side material rules against the reference's own unit checks (V13, src/core/15-verify.js:
420-446): the Cu-pattern mixing rules of a substrate row with V13's inputs (Cu 110 GPa, nu 0.34,
16.4 ppm; matrix 10 GPa, nu 0.30, 20 ppm; r = 0.5, signal layer) to 1e-9, and the rotated cubic
stiffness of (100) silicon: 169 GPa along the die edge <110> (1e-3) and 130 GPa along the
diagonal <100> (1.1e-3), V13's rounded references and tolerances."""
import numpy as np

from tmsolve.materials import directional_modulus, iso_ec, mix_cu_ec, silicon_d, substrate_row_ec


def test_v13_mixing_rules():
    cu, d = iso_ec(110000, 0.34, 16.4e-6), iso_ec(10000, 0.30, 20e-6)
    m = mix_cu_ec(cu, d, 0.5, "signal")
    turner = (0.5 * 110000 * 16.4e-6 + 0.5 * 10000 * 20e-6) / (0.5 * 110000 + 0.5 * 10000)
    assert abs(m["ax"] / turner - 1) <= 1e-9
    assert abs(m["Ez"] / (0.5 * 110000 + 0.5 * 10000) - 1) <= 1e-9
    assert abs(m["Ex"] / (0.5 * (60000 + 1 / (0.5 / 110000 + 0.5 / 10000))) - 1) <= 1e-9
    # a plane layer mixes in-plane by Voigt too
    p = mix_cu_ec(cu, d, 0.5, "plane")
    assert abs(p["Ex"] - 60000) <= 1e-9 * 60000


def test_v13_silicon_moduli():
    D = silicon_d("aniso")
    assert abs(directional_modulus(D, [1, 0, 0]) / 1000 / 169 - 1) <= 1e-3
    assert abs(directional_modulus(D, [np.sqrt(0.5), np.sqrt(0.5), 0]) / 1000 / 130 - 1) <= 1.1e-3
    # the isotropic option is 130 GPa in every direction
    assert abs(directional_modulus(silicon_d("iso"), [1, 0, 0]) - 130e3) <= 1e-6 * 130e3


def test_substrate_rows():
    mats = dict(cu=iso_ec(110000, 0.34, 16.4e-6), diel=iso_ec(5000, 0.34, 40e-6), core=iso_ec(28000, 0.2, 12e-6),
                sr=iso_ec(3000, 0.35, 50e-6))
    assert substrate_row_ec(dict(type="sr", mat="sr"), mats)["Ex"] == 3000
    sig = substrate_row_ec(dict(type="cu", r=0.45, kind="signal", fill="diel"), mats)
    pla = substrate_row_ec(dict(type="cu", r=0.45, kind="plane", fill="diel"), mats)
    assert sig["Ez"] == pla["Ez"] and sig["Ex"] < pla["Ex"]        # Voigt through the thickness; Reuss lowers the signal layer
    core = substrate_row_ec(dict(type="core", mat="core", pth=0.02), mats)
    assert abs(core["Ex"] - (0.02 * 110000 + 0.98 * 28000)) <= 1e-9 * core["Ex"]
