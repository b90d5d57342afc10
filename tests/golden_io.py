"""Load the golden fixtures written by tests/golden/make_golden.py."""
import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def load_case(path):
    d = np.load(path, allow_pickle=True)
    dim = str(d["dim"])
    name = os.path.splitext(os.path.basename(path))[0]
    out, in_ = eval(str(d["request"]), {"array": np.array})  # fixtures are written by our own script
    bc = d["bc"]
    bc = str(bc) if bc.dtype == object else (float(bc) if bc.ndim == 0 else [float(x) for x in bc])
    case = {"name": name, "dim": dim, "S": d["S"], "out": out, "in": in_, "eps_checksum": d["eps_checksum"]}
    syst = {"epsilon_L": complex(d["epsilon_L"]), "epsilon_R": complex(d["epsilon_R"]), "k0dx": complex(d["k0dx"])}
    for k in ("epsilon_L", "epsilon_R", "k0dx"):
        if syst[k].imag == 0:
            syst[k] = syst[k].real
    syst["yBC" if dim == "2d" else "xyBC"] = bc
    if "epsilon" in d:
        syst["epsilon"] = d["epsilon"]
    case["syst"] = syst
    for side in ("L", "R"):
        case[f"N_prop_{side}"] = int(d[f"N_prop_{side}"])
        case[f"ind_prop_{side}"] = d[f"ind_prop_{side}"]
        case[f"sqrt_mu_{side}"] = d[f"sqrt_mu_{side}"]
        case[f"kx_{side}"] = d[f"kx_{side}"]
    return case


def config_case(name):
    """Golden record of a seeded config, with its syst regenerated."""
    from rgf_b200 import workloads
    path = os.path.join(GOLDEN, f"{name}.npz")
    if not os.path.exists(path):
        return None
    case = load_case(path)
    if name.startswith("cfg4_"):
        k = int(name.split("_")[1])
        syst, out, in_ = workloads.config4_structure(k)
    else:
        syst, out, in_ = getattr(workloads, "config" + name[3:])()
    case["syst"] = syst
    return case
