"""Generate tests/golden/exchange_map.json: which partner cell feeds each ghost cell of
an ExchangeBC_FullFace, for every face pair and orientation, read from the reference's
source text (run from the repository root: python tests/golden/make_exchange_map.py
[path to the reference checkout]).

The reference sets the mapping up in GhostCellFullFaceCopy.set_up_cell_mapping_phase0
(src/eilmer/bc/ghost_cell_effect/full_face_copy.d:680-1409): for the ghost cell at
depth n (0 = next to the face) beyond face `which_boundary` at this block's tangential
indices, the source is other_blk.cell_index(i_src, j_src, k_src) with each index
either a constant face index (0 or n?c - 1) moved n cells into the partner, or one of
this block's loop indices, possibly reversed (n?c - x - 1).  2D blocks have one table
(orientation ignored), 3D blocks one per orientation 0..3.

Output: a list of records {dims, face, other_face, orientation, src}, faces numbered as
this library numbers them (0 west/i-, 1 east/i+, 2 south/j-, 3 north/j+, 4 bottom/k-,
5 top/k+), src[d] = [sel, flip] for the partner's index along axis d: sel 0, 1, 2 =
this block's i, j, k; sel 3 = the ghost's depth n; flip 1 = counted from the partner's
far end (n_d - 1 - value).  In 2D src[2] is [2, 0] (k = 0 on both sides).
"""
import json
import os
import re
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REF = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("GDTK_REFERENCE", "/root/reference")
SRC = os.path.join(REF, "src", "eilmer", "bc", "ghost_cell_effect", "full_face_copy.d")

# Eilmer's Face enum names -> this library's face numbers
FACE = {"west": 0, "east": 1, "south": 2, "north": 3, "bottom": 4, "top": 5}
AX = "ijk"


def parse(text):
    """(dims, face, other_face, orientation or None) -> {axis letter: expression}, and the
    partner cell expression 'i_src,j_src-n,k_src' per (dims, face, other_face)."""
    lines = text.split("\n")
    start = next(n for n, ln in enumerate(lines) if "void set_up_cell_mapping_phase0()" in ln)
    end = next(n for n in range(start + 1, len(lines)) if re.match(r"\s*void set_up_cell_mapping_phase1", lines[n]))
    dims, this, other = None, None, None
    tang, cell = {}, {}
    for ln in lines[start:end]:
        s = ln.strip()
        if "dimensions == 2" in s:
            dims = 2
        if s.startswith("// presume dimensions == 3"):
            dims = 3
        m = re.match(r"case Face\.(\w+):", s)
        if m:
            indent = len(ln) - len(ln.lstrip())
            if indent <= 12:
                this, other = m.group(1), None
            else:
                other = m.group(1)
            continue
        m = re.match(r"case (\d): (.*)", s)
        if m and dims == 3:
            for ax, ex in re.findall(r"([ijk])_src = ([^;]+);", m.group(2)):
                tang.setdefault((3, this, other, int(m.group(1))), {})[ax] = ex.strip()
            continue
        for ax, ex in re.findall(r"\b([ijk])_src = ([^;]+);", s):
            if this and other:
                tang.setdefault((dims, this, other, None), {})[ax] = ex.strip()
        m = re.search(r"mapped_cell_ids ~= other_blk\.cell_index\(([^)]*)\)", s)
        if m and this and other:
            cell[(dims, this, other)] = [e.strip() for e in m.group(1).split(",")]
    return tang, cell


def term(ex, ax):
    """[sel, flip] of one tangential or normal index expression."""
    ex = ex.replace(f"other_blk.n{ax}c", "N")
    if ex in ("i", "j", "k"):
        return [AX.index(ex), 0]
    m = re.fullmatch(r"N - ([ijk]) - 1", ex)
    if m:
        return [AX.index(m.group(1)), 1]
    if ex == "0":
        return [3, 0]
    if ex == "N - 1":
        return [3, 1]
    raise ValueError(f"unexpected index expression {ex!r}")


def main():
    tang, cell = parse(open(SRC).read())
    out = []
    for (dims, this, other, o), t in sorted(tang.items(), key=lambda kv: (kv[0][0], FACE[kv[0][1]], FACE[kv[0][2]],
                                                                        -1 if kv[0][3] is None else kv[0][3])):
        if dims == 3 and o is None:
            continue   # the normal index alone; merged below
        full = dict(t)
        if dims == 3:
            full.update(tang[(3, this, other, None)])
        src = []
        for d in range(3 if dims == 3 else 2):
            ax = AX[d]
            sel, flip = term(full[ax], ax)
            if sel == 3:   # the partner's face index: the ghost at depth n sits n cells inside it
                want = f"{ax}_src-n" if flip else f"{ax}_src+n"
                assert cell[(dims, this, other)][d] == want, (this, other, cell[(dims, this, other)])
            src.append([sel, flip])
        if dims == 2:
            src.append([2, 0])
        out.append({"dims": dims, "face": FACE[this], "other_face": FACE[other],
                    "orientation": 0 if o is None else o, "src": src})
    assert len(out) == 16 + 144, len(out)
    with open(os.path.join(HERE, "exchange_map.json"), "w") as f:
        json.dump({"source": "src/eilmer/bc/ghost_cell_effect/full_face_copy.d:680-1409", "maps": out}, f,
                  separators=(",", ":"))
    print(f"{len(out)} face-pair maps")


if __name__ == "__main__":
    main()
