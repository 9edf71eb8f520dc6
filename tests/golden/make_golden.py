"""Extract the reference's known-answer vectors for the APIC / PolyPIC tests.

The reference's unit tests (``unit_test/tstAPIC.hpp``, ``unit_test/tstPolyPIC.hpp``)
hold Mathematica-computed values for a single-particle fixture: grid values,
g2p particle velocity / affine matrix / polynomial modes, p2g grid momentum
and grid mass.  This script reads those two files as text and writes the
numbers into ``apic_polypic_golden.json`` next to it, together with the
fixture parameters parsed from the same files (mesh box, cell size, halo
width, particle mass/position/cell, time step, tolerance).

It only runs where the reference tree is present; the JSON it produced is
committed and is what the tests read.

Usage:  python tests/golden/make_golden.py REFERENCE_ROOT
        (or PICASSO_REFERENCE_ROOT=... python tests/golden/make_golden.py)
"""

import json
import os
import re
import sys

CHECKS = ("checkGridVelocity", "checkParticleVelocity", "checkGridMomentum",
          "checkGridMass", "setParticleVelocity")

_func_re = re.compile(
    r"void\s+(" + "|".join(CHECKS) + r")\s*\(\s*std::integral_constant<int,\s*(\d)>")
_arr_re = re.compile(r"double\s+(\w+)((?:\[\d+\])+)\s*=\s*\{(.*?)\};", re.S)
_num_re = re.compile(r"[-+]?(?:\d+\.\d*|\.\d+|\d+)(?:[eE][-+]?\d+)?")


def _reshape(flat, dims):
    if len(dims) == 1:
        assert len(flat) == dims[0], (len(flat), dims)
        return flat
    step = len(flat) // dims[0]
    return [_reshape(flat[i * step:(i + 1) * step], dims[1:]) for i in range(dims[0])]


def parse_checks(text):
    """Return {order: {function: {array_name: nested list}}}."""
    out = {}
    starts = [(m.start(), m.group(1), int(m.group(2))) for m in _func_re.finditer(text)]
    for n, (pos, fname, order) in enumerate(starts):
        end = starts[n + 1][0] if n + 1 < len(starts) else len(text)
        body = text[pos:end]
        arrays = {}
        for am in _arr_re.finditer(body):
            dims = [int(d) for d in re.findall(r"\[(\d+)\]", am.group(2))]
            flat = [float(v) for v in _num_re.findall(am.group(3))]
            arrays[am.group(1)] = _reshape(flat, dims)
        out.setdefault(order, {})[fname] = arrays
    return out


def parse_fixture(text):
    def num(name):
        m = re.search(r"\b" + name + r"\s*=\s*([-+0-9.eE]+)\s*;", text)
        return float(m.group(1)) if m else None
    fx = {k: num(k) for k in ("pm", "px", "py", "pz", "dt", "near_eps")}
    for k in ("cx", "cy", "cz"):
        fx[k] = int(num(k))
    box = re.search(r"global_box\s*=\s*\{([^}]*)\}", text)
    fx["global_box"] = [float(v) for v in _num_re.findall(box.group(1))]
    return {k: v for k, v in fx.items() if v is not None}


def main():
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("PICASSO_REFERENCE_ROOT")
    if not ref:
        sys.exit("usage: make_golden.py <Picasso source tree> "
                 "(or set PICASSO_REFERENCE_ROOT)")
    ut = os.path.join(ref, "unit_test")
    out = {"source": "reference unit_test/tstAPIC.hpp and unit_test/tstPolyPIC.hpp "
                     "(Mathematica-generated known answers)"}
    for name, fname in (("apic", "tstAPIC.hpp"), ("polypic", "tstPolyPIC.hpp")):
        with open(os.path.join(ut, fname)) as f:
            text = f.read()
        out[name] = {"checks": parse_checks(text), "fixture": parse_fixture(text)}
    with open(os.path.join(ut, "inputs", "polypic_test.json")) as f:
        mesh = json.load(f)["mesh"]
    out["mesh_input"] = mesh
    here = os.path.dirname(os.path.abspath(__file__))
    path = os.path.join(here, "apic_polypic_golden.json")
    with open(path, "w") as f:
        json.dump(out, f, indent=1)
    print("wrote", path)


if __name__ == "__main__":
    main()
