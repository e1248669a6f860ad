"""Extract the reference's logged known answers for the MHD step into known_answers.json.

Reads the reference's recorded CPU validation log (docs/data/validation-cpu.log of
yipihey/pmf-glm, produced by test/inherited/runtests.jl) and the CT/CFL expectations
written in its tests. Run once in a container where the reference checkout exists:

    python tests/golden/make_known_answers.py /path/to/pmf-glm
"""
import json
import os
import re
import sys

if len(sys.argv) != 2:
    sys.exit("usage: python tests/golden/make_known_answers.py <path to the pmf-glm checkout>")
ref = sys.argv[1]
log = open(os.path.join(ref, "docs/data/validation-cpu.log")).read()
out = {"source": "docs/data/validation-cpu.log (test/inherited/runtests.jl)", "alfven": {}}
for recon in ("plm", "ppm"):
    for m in re.finditer(r"\[%s\] N=(\d+)\s+L1\(By\)=([0-9.e+-]+).*?\((\d+) steps" % recon, log):
        out["alfven"]["%s_%s" % (recon, m.group(1))] = {"L1": float(m.group(2)), "steps": int(m.group(3))}
m = re.search(r"low-beta Alfv.n t=[0-9.]+ \((\d+) steps\): L1\(By\)=([0-9.e+-]+)", log)
out["alfven_lowbeta_64"] = {"L1": float(m.group(2)), "steps": int(m.group(1))}
m = re.search(r"Brio-Wu t=[0-9.]+: .*?min=([0-9.]+) max=([0-9.]+) \| L1\(256 vs 512\)=([0-9.e+-]+)", log)
out["brio_wu"] = {"rho_min": float(m.group(1)), "rho_max": float(m.group(2)), "L1_256_vs_512": float(m.group(3))}
m = re.search(r"OT t=[0-9.]+ \((\d+) steps\): .*?max\|divB\|.dx/Brms=([0-9.]+)", log)
out["orszag_tang_128"] = {"steps": int(m.group(1)), "divb_dx_over_brms": float(m.group(2))}
# tolerances of the reference's parity gates (test/test_backends.jl:65-72,118)
out["parity"] = {"rtol": 5e-5, "atol": 2e-6, "mass_drift": 3e-6}
# CT fork-port agreement (test/inherited/test_ct.jl:209-241)
out["ct_fork_port"] = {"N": 12, "steps": 5, "cfl": 0.3, "rel_tol": 1e-10}
json.dump(out, open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "known_answers.json"), "w"), indent=1)
print(json.dumps(out, indent=1))
