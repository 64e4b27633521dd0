"""Extract the golden values printed by the reference's own notebooks.

The reference (cabrer7/PyWignerCUDA2) ships no tests; the only recorded
outputs of its code path are the notebook cells under ``instances/``.  The
Dirac and KvN notebooks print the trace norm before every renormalisation
(``Normalize_4x4_GPU``, GPU_WignerDirac4D.py:1366-1369): once after the
initial condition and once per ``Run()`` iteration.  This script reads those
notebooks as text and writes ``notebook_norms.json`` beside itself.

Run it where the reference tree is mounted::

    python tests/golden/make_golden.py /root/reference

It is the only file in this repository that reads the reference tree; the
JSON it writes is committed and is what the tests use.
"""
import json
import os
import re
import sys

NOTEBOOKS = [
    "instances/WignerDirac4D_64_64/Free.ipynb",
    "instances/WignerDirac4D_64_64/FreeFiltered.ipynb",
    "instances/WignerDirac4D_64_64/Landao.ipynb",
    "instances/WignerDirac4D_64_64/Landao_X.ipynb",
    "instances/WignerDirac4D_64_64/SternGerlach.ipynb",
    "instances/WignerDirac4D_64_64/X.ipynb",
    "instances/WignerDirac4D_64_64/X2.ipynb",
    "instances/WignerDirac4D_64_64/X_Filtered.ipynb",
    "instances/WignerDirac4D_64_64/Y.ipynb",
    "instances/WignerDiracKvN4D_64_64/Free_Vx.ipynb",
    "instances/WignerDiracKvN4D_64_64/Free_Vy.ipynb",
]

NORM_RE = re.compile(r"\(\s*([-+0-9.eE]+)\s*([-+][0-9.eE]+)j\)")


def _cells(nb):
    sheets = nb["worksheets"] if "worksheets" in nb else [nb]
    for sheet in sheets:
        for cell in sheet["cells"]:
            if cell["cell_type"] == "code":
                yield cell


def _text(cell):
    return "".join("".join(o.get("text", [])) for o in cell.get("outputs", []))


def extract(path):
    nb = json.load(open(path))
    out = {"init_norms": [], "run_norms": [], "final_trace_norm": None,
           "running_time_min": None}
    for cell in _cells(nb):
        src = "".join(cell.get("input", cell.get("source", [])))
        text = _text(cell)
        norms = [complex(float(a), float(b)) for a, b in NORM_RE.findall(text)]
        if "Set_Initial_Condition" in src and "def " not in src:
            out["init_norms"] += [n.real for n in norms]
        elif "instance.Run()" in src:
            out["run_norms"] += [n.real for n in norms]
            m = re.search(r"running time =\s*([0-9.eE+-]+)", text.replace("\n", " "))
            if m:
                out["running_time_min"] = float(m.group(1))
        elif "np.sum(W_end)" in src:
            m = re.search(r"([-+]?[0-9]+\.[0-9]+(?:[eE][-+]?[0-9]+)?)", text)
            if m:
                out["final_trace_norm"] = float(m.group(1))
    return out


def main(root):
    result = {}
    for rel in NOTEBOOKS:
        result[rel] = extract(os.path.join(root, rel))
    dst = os.path.join(os.path.dirname(os.path.abspath(__file__)), "notebook_norms.json")
    with open(dst, "w") as f:
        json.dump(result, f, indent=1, sort_keys=True)
    for k, v in result.items():
        print(k, len(v["init_norms"]), len(v["run_norms"]), v["final_trace_norm"],
              v["running_time_min"])


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: make_golden.py <path of the cabrer7/PyWignerCUDA2 checkout>")
    main(sys.argv[1])
