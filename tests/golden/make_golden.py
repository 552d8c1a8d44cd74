"""Generate the golden fixtures of this directory from the GridSim reference tree.

Run in a container that holds the reference source (argument: its root). It writes, for each
bundled MATPOWER case the reference's own tests use, the parsed model (``gridsim_b200.model.parse_matpower``,
the restatement of ``IO/Matpower/MatpowerParser.cs``) and the published solved voltages the reference
tests pin:

* case9: ``tests/GridSim.Tests/PowerFlowTests.cs:11-15`` (ExpectedVm / ExpectedVaDeg, tolerances :38-46);
* case14/57/118/300: ``tests/GridSim.Tests/IeeeCasesTests.cs:16-24`` arrays, tolerances :91-95.

The fixtures are what the tests read; the tests never read the reference tree.
"""
import json
import os
import re
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
from gridsim_b200.model import load_matpower  # noqa: E402


def arrays(cs_text):
    out = {}
    for m in re.finditer(r"double\[\]\s+(\w+)\s*=\s*\{([^}]*)\}", cs_text, re.S):
        out[m.group(1)] = [float(v) for v in m.group(2).replace("\n", " ").split(",") if v.strip()]
    return out


def main(ref_root):
    tests = os.path.join(ref_root, "tests", "GridSim.Tests")
    pf = arrays(open(os.path.join(tests, "PowerFlowTests.cs")).read())
    ieee = arrays(open(os.path.join(tests, "IeeeCasesTests.cs")).read())
    published = {
        "case9": (pf["ExpectedVm"], pf["ExpectedVaDeg"], 1e-3, 1e-2),   # Assert.Equal(..., 3) / (..., 2)
        "case14": (ieee["Case14Vm"], ieee["Case14Va"], 0.005, 0.2),
        "case57": (ieee["Case57Vm"], ieee["Case57Va"], 0.02, 1.5),
        "case118": (ieee["Case118Vm"], ieee["Case118Va"], 0.03, 1.0),
        "case300": (ieee["Case300Vm"], ieee["Case300Va"], 0.02, 12.0),
    }
    for name, (vm, va, vm_tol, va_tol) in published.items():
        m = load_matpower(os.path.join(ref_root, "data", "matpower", "lib", name + ".m"))
        doc = {"source": f"data/matpower/lib/{name}.m", "model": m.to_dict(),
               "published": {"vm": vm, "va_deg": va, "vm_tol": vm_tol, "va_tol_deg": va_tol}}
        with open(os.path.join(HERE, name + ".json"), "w") as fh:
            json.dump(doc, fh)
        print(name, m.n_bus, "buses", m.n_branch, "branches", m.n_gen, "gens")


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")
