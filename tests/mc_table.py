"""Reads the marching-cubes table committed in sesmesh_b200/csrc/mc_table.inc."""
import os
import re

_INC = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "sesmesh_b200", "csrc",
                    "mc_table.inc")


def load():
    text = open(_INC).read()
    off = re.search(r"SMB_TRI_OFFSET\[257\] = \{(.*?)\};", text, re.S).group(1)
    offsets = [int(v) for v in re.findall(r"\d+", off)]
    body = re.search(r"SMB_TRI_EDGES\[\d+\]\[3\] = \{(.*?)\};", text, re.S).group(1)
    body = re.sub(r"//[^\n]*", "", body)
    tris = [tuple(int(v) for v in t) for t in re.findall(r"\{(\d+), (\d+), (\d+)\}", body)]
    return offsets, tris


EDGE_LOWER = [[0, 2, 4, 6], [0, 1, 4, 5], [0, 1, 2, 3]]


def edge_corners(e):
    axis, lo = e // 4, EDGE_LOWER[e // 4][e % 4]
    return lo, lo | (1 << axis)
