"""Parse the reference's shipped trace files -- the robot-arm traces
src/models/robotarm/input_ra, input1, input2, input5 (each line: x y
angles[5] controls[5] dt actual_x actual_y actual_angles[5]) and the unicycle
program's src/models/unicycle/input (ranges[10] v omega dt x y theta) -- into
FP32 arrays, token by token with the C library's strtof (the value the
drivers' fscanf("%f") reads), and store them in ref_traces.npz beside this
script.  The GPU tests write them back as text with 9 significant digits
(which reads back as the same FP32 values) and run both the engine's and the
reference's drivers on them.  Needs the reference tree ($ESTHERA_REF, else
../reference beside the repository)."""
import ctypes as C
import os
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REF = Path(os.environ.get("ESTHERA_REF", HERE.parents[2] / "reference"))
FILES = {"robotarm_input_ra": "src/models/robotarm/input_ra", "robotarm_input1": "src/models/robotarm/input1",
         "robotarm_input2": "src/models/robotarm/input2", "robotarm_input5": "src/models/robotarm/input5",
         "unicycle_input": "src/models/unicycle/input"}


def main():
    libc = C.CDLL(None)
    libc.strtof.restype = C.c_float
    libc.strtof.argtypes = [C.c_char_p, C.c_void_p]
    out = {}
    for key, rel in FILES.items():
        rows = []
        for line in (REF / rel).read_text().splitlines():
            tok = line.split()
            if tok:
                rows.append([libc.strtof(t.encode(), None) for t in tok])
        out[key] = np.array(rows, np.float32)
    np.savez_compressed(HERE / "ref_traces.npz", **out)
    print("wrote", HERE / "ref_traces.npz", {k: v.shape for k, v in out.items()})


if __name__ == "__main__":
    main()
