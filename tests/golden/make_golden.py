"""Write the crafted-plane golden vectors of the reference's device tests.

Restates the planes of test/test_ka.jl:51-70 (stillyslalom/Hammerhead.jl) and
the answers find_peaks(R, 4; peak_finder = :regionalmax) gives for them under
the reference's rules (src/correlators.jl:426-454, src/localmax.jl:3-19):
regional maxima with ties going to the later column-major point on a plateau,
equal distinct maxima ordered by earlier column-major index, a non-positive
primary allowed but secondaries required positive, NaN never a maximum.
Locations are 1-based (row, col). Run: python tests/golden/make_golden.py
"""
import json
import math
import os

HERE = os.path.dirname(os.path.abspath(__file__))


def zeros(nr, nc, val=0.0):
    return [[val] * nc for _ in range(nr)]


def main():
    nearby = zeros(16, 16)
    nearby[7][7] = 1.0     # R[8, 8]
    nearby[7][8] = 0.1     # R[8, 9]
    nearby[7][9] = 0.8     # R[8, 10]: distinct maximum inside the exclusion radius
    nearby[4][2] = 0.6     # R[5, 3]
    nearby[11][12] = 0.6   # R[12, 13]: equal value, earlier column-major point wins
    plateau = zeros(7, 9, 1.0)
    nonpositive = zeros(8, 8, -2.0)
    nonpositive[2][3] = -1.0  # R[3, 4]
    allnan = zeros(8, 8, float("nan"))
    cases = {
        "nearby": dict(plane=nearby, k=4, values=[1.0, 0.8, 0.6, 0.6],
                       locations=[[8, 8], [8, 10], [5, 3], [12, 13]]),
        "plateau": dict(plane=plateau, k=4, values=[1.0], locations=[[7, 9]]),
        "nonpositive": dict(plane=nonpositive, k=4, values=[-1.0], locations=[[3, 4]]),
        "allnan": dict(plane=allnan, k=4, values=[], locations=[]),
    }
    with open(os.path.join(HERE, "crafted_planes.json"), "w") as f:
        json.dump(cases, f, indent=1, allow_nan=True)


if __name__ == "__main__":
    main()
