"""Extract the reference's golden norms into tests/golden/reference_logs.json.

Usage: python tests/golden/make_golden.py <path to a MeltPoolDG source tree>.  The output is
committed so that nothing at test time reads the reference tree.

Sources (paths inside the MeltPoolDG tree):
  applications/mp-heat-transfer/cases/unidirectional_heat_transfer/tests/
      unidirectional_heat_transfer.mpirun=4.output   (Newton "||solution||" per step)
  applications/mp-advec-diff/cases/tests/advection_diffusion_vortex_mf_3d.mpirun=4.output
  applications/mp-advec-diff/cases/tests/advection_diffusion_vortex_mf.mpirun=4.output
  applications/mp-advec-diff/cases/tests/advection_diffusion_vortex_mf_inflow_outflow{,_3d}.mpirun=4.output
  applications/mp-advec-diff/cases/tests/advection_diffusion_vortex_mf_supg.mpirun=4.output
      ("|| advected field ||L2" per step)
"""
import json
import os
import re
import sys

if len(sys.argv) != 2:
    sys.exit("usage: make_golden.py <path to a MeltPoolDG source tree>")
REF = sys.argv[1]
CASES = {
    "heat_unidirectional_2d_q1": (
        "applications/mp-heat-transfer/cases/unidirectional_heat_transfer/tests/"
        "unidirectional_heat_transfer.mpirun=4.output",
        r"\|\|solution\|\| = ([0-9.eE+-]+)"),
    "advdiff_vortex_mf_3d_q1": (
        "applications/mp-advec-diff/cases/tests/advection_diffusion_vortex_mf_3d.mpirun=4.output",
        r"\|\| advected field \|\|L2 = ([0-9.eE+-]+)"),
    "advdiff_vortex_mf_2d_q1": (
        "applications/mp-advec-diff/cases/tests/advection_diffusion_vortex_mf.mpirun=4.output",
        r"\|\| advected field \|\|L2 = ([0-9.eE+-]+)"),
    "advdiff_vortex_mf_inflow_outflow_3d_q1": (
        "applications/mp-advec-diff/cases/tests/advection_diffusion_vortex_mf_inflow_outflow_3d.mpirun=4.output",
        r"\|\| advected field \|\|L2 = ([0-9.eE+-]+)"),
    "advdiff_vortex_mf_inflow_outflow_2d_q1": (
        "applications/mp-advec-diff/cases/tests/advection_diffusion_vortex_mf_inflow_outflow.mpirun=4.output",
        r"\|\| advected field \|\|L2 = ([0-9.eE+-]+)"),
    "advdiff_vortex_supg_2d_q1": (
        "applications/mp-advec-diff/cases/tests/advection_diffusion_vortex_mf_supg.mpirun=4.output",
        r"\|\| advected field \|\|L2 = ([0-9.eE+-]+)"),
}

out = {}
for name, (rel, pat) in CASES.items():
    text = open(os.path.join(REF, rel)).read()
    out[name] = {"source": rel, "values": [v for v in re.findall(pat, text)]}
path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "reference_logs.json")
with open(path, "w") as f:
    json.dump(out, f, indent=1)
print(path)
