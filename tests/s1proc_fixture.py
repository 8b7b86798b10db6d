"""Records of tests/golden/s1proc_pins.npz (outputs of the reference's own
Python for amplitude looks, coherence and stitching; made by
tests/golden/make_s1proc_golden.py)."""
import os

import numpy as np

PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "s1proc_pins.npz")


def load():
    return np.load(PATH)


def looks_cases(z):
    k = 0
    while f"looks{k}_in" in z:
        rl, cl = (int(v) for v in z[f"looks{k}_rc"])
        yield z[f"looks{k}_in"], rl, cl, z[f"looks{k}_cpx"], z[f"looks{k}_pow"]
        k += 1


def multilook_bursts(z):
    out, i = [], 0
    while f"ml_burst{i}_hdr" in z:
        out.append((z[f"ml_burst{i}_hdr"], z[f"ml_burst{i}_data"]))
        i += 1
    return out


ML_LOOKS = ((2, 4), (1, 1), (3, 8))


def stitch_bursts(z):
    """[(header, data, subswath, group)]; group: the pair of product ids the
    reference reads from file-name words 1+2 and 7+8 (interfere.py:92-96)."""
    groups, out = {}, []
    for k, name in enumerate(z["st_names"]):
        w = str(name).split("_")
        g = groups.setdefault((w[1] + w[2], w[7] + w[8]), len(groups))
        sw = int(z[f"st_burst{k}_meta"][0])
        out.append((z[f"st_burst{k}_hdr"], z[f"st_burst{k}_data"], sw, g))
    return out
