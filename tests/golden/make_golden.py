"""Generate the golden fixtures of this directory from the GridSim reference tree.

Run in a container that holds the reference source (argument: its root). It writes, for each
bundled MATPOWER case the reference's own tests use, the parsed model (``gridsim_b200.model.parse_matpower``,
the restatement of ``IO/Matpower/MatpowerParser.cs``) and the published solved voltages the reference
tests pin:

* case9: ``tests/GridSim.Tests/PowerFlowTests.cs:11-15`` (ExpectedVm / ExpectedVaDeg, tolerances :38-46);
* case14/57/118/300: ``tests/GridSim.Tests/IeeeCasesTests.cs:16-24`` arrays, tolerances :91-95.

It also turns the reference's captured ``gridsim nminus1`` outputs
(``tests/GridSim.Tests/fixtures/cli-stdout/nminus1-*.txt``: every outage's status, maximum loading, worst boundary
loading and voltage extremes, after netting against the base case) and ``gridsim nminus2`` outputs (``nminus2-*.txt``:
the worst pairs, the count line and the single outages left out of the pairing) into ``cli_nminus1.json``.

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
    # case24_ieee_rts: the model only, for its RATE_B / RATE_C columns
    # (tests/GridSim.Tests/ContingencyTypesAndRatingsTests.cs:43-51)
    m24 = load_matpower(os.path.join(ref_root, "data", "matpower", "lib", "case24_ieee_rts.m"))
    with open(os.path.join(HERE, "case24_ieee_rts.json"), "w") as fh:
        json.dump({"source": "data/matpower/lib/case24_ieee_rts.m", "model": m24.to_dict(), "published": None}, fh)
    for name, (vm, va, vm_tol, va_tol) in published.items():
        m = load_matpower(os.path.join(ref_root, "data", "matpower", "lib", name + ".m"))
        doc = {"source": f"data/matpower/lib/{name}.m", "model": m.to_dict(),
               "published": {"vm": vm, "va_deg": va, "vm_tol": vm_tol, "va_tol_deg": va_tol}}
        with open(os.path.join(HERE, name + ".json"), "w") as fh:
            json.dump(doc, fh)
        print(name, m.n_bus, "buses", m.n_branch, "branches", m.n_gen, "gens")


def parse_cli_screen(text):
    """One captured N-1 table: the base-case line, each outage row, and the 'makes ... worse' notes."""
    lines = text.replace("\r\n", "\n").split("\n")
    out = {"base": None, "rows": [], "worsened": {}}
    in_table = False
    for ln in lines:
        if ln.startswith("Base case: secure"):
            out["base"] = []
        elif ln.startswith("Base case:"):
            out["base"] = [t.strip() for t in ln.split("any outage:", 1)[1].split(";")]
        elif ln.startswith("Outage "):
            in_table = True
        elif ln.startswith("-----"):
            if in_table and out["rows"]:
                in_table = False
        elif in_table and ln.strip():
            label, rest = ln[:30].strip(), ln[32:]
            status, tail = rest[:12].strip(), rest[14:].strip()
            m = re.match(r"(\d+)%\s+(\d+)%\s+([0-9.]+)\s+([0-9.]+)$", tail)
            row = {"outage": label, "status": status}
            if m:
                row.update(max_load=int(m.group(1)), worst_bnd=int(m.group(2)), vmin=m.group(3), vmax=m.group(4))
            else:
                row["text"] = tail
            out["rows"].append(row)
        elif ln.startswith("  ") and ": makes base-case violation(s) worse: " in ln:
            who, what = ln.strip().split(": makes base-case violation(s) worse: ")
            out["worsened"][who] = [t.strip() for t in what.split(";")]
    return out


def cli_screens(ref_root):
    fx = os.path.join(ref_root, "tests", "GridSim.Tests", "fixtures", "cli-stdout")
    doc = {}
    for name, case, per_bus in (("nminus1-case9", "case9", True), ("nminus1-case9-global-vlimits", "case9", False),
                                ("nminus1-case14", "case14", True)):
        d = parse_cli_screen(open(os.path.join(fx, name + ".txt")).read())
        d.update(case=case, per_bus_voltage_limits=per_bus, source=f"tests/GridSim.Tests/fixtures/cli-stdout/{name}.txt")
        doc[name] = d
        print(name, len(d["rows"]), "rows")
    for name, case, per_bus in (("nminus2-case9", "case9", True), ("nminus2-case9-global-vlimits", "case9", False)):
        text = open(os.path.join(fx, name + ".txt")).read()
        d = parse_cli_screen(text)
        m = re.search(r"\(showing worst (\d+) of (\d+)\)", text)
        d["screened"] = int(m.group(2)) if m else len(d["rows"])
        m = re.search(r"(\d+) outages screened\s+(\d+) secure\s+(\d+) with violations\s+(\d+) islanded", text)
        d["counts"] = [int(m.group(i)) for i in range(1, 5)]
        d["excluded"] = [[ln[:32].strip(), ln[32:].strip()] for ln in text.split("\n")[text.split("\n").index(
            next(ln for ln in text.split("\n") if "left out of the pairing" in ln)) + 1:] if ln.startswith("  ")]
        d.update(case=case, per_bus_voltage_limits=per_bus, k=2, candidate_count=20,
                 source=f"tests/GridSim.Tests/fixtures/cli-stdout/{name}.txt")
        doc[name] = d
        print(name, d["screened"], "combinations")
    with open(os.path.join(HERE, "cli_nminus1.json"), "w") as fh:
        json.dump(doc, fh, indent=1)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_golden.py <root of the GridSim source tree>")
    root = sys.argv[1]
    main(root)
    cli_screens(root)
