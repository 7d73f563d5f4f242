"""Shared fixtures-free helpers for the tests (geometry builders that mirror
the reference's test geometries)."""
import numpy as np

from gpurify_b200.geometry import Deck, GeometryStore, PexLayerParams


def bridge_test_deck(method="field_solver"):
    """crates/pex/tests/bridge.rs:8-43: met1 (sheet 0.1, t 200 nm, h 500 nm,
    k 3.9) and via1 (fixed 5 ohm)."""
    return Deck.from_dict({
        "layers": {"met1": {"layer": 68, "datatype": 20}, "via1": {"layer": 67, "datatype": 44}},
        "pex_method": method,
        "pex": {
            "met1": {"sheet_res_ohm_sq": 0.1, "area_cap_af_um2": 25.0, "fringe_cap_af_um": 40.0,
                     "coupling_cap_af_um": 100.0, "coupling_ref_spacing_nm": 200.0, "thickness_nm": 200.0,
                     "height_nm": 500.0, "dielectric_k": 3.9},
            "via1": {"sheet_res_ohm_sq": 0.0, "area_cap_af_um2": 0.0, "fringe_cap_af_um": 0.0,
                     "coupling_cap_af_um": 0.0, "coupling_ref_spacing_nm": 1.0, "via_res_ohm": 5.0,
                     "thickness_nm": 200.0, "height_nm": 300.0, "dielectric_k": 3.9},
        },
    })


def rel_max(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))
