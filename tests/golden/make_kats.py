"""Extract the reference's known-answer values into reference_kats.json.

Reads the literal inputs and expected outputs of the reference's own unit
tests (run where the reference repository is available; the JSON it writes
is committed so the tests need no reference checkout):

  crates/pippin/src/newton.rs   impedance_curve          (impedance KAT)
  crates/pippin/src/math.rs     block_cholesky_matches_dense_on_block_diagonal,
                                cholesky_solves, quat_mat_roundtrip
  crates/pippin/src/simd.rs     dot_matches_scalar
  crates/pippin/src/mesh.rs     cube_mass_properties_are_exact

Each entry records the file and line the values were read from.
"""
import json
import os
import re
import sys

REF = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("PIPPIN_REFERENCE", "")
if not REF:
    sys.exit("usage: make_kats.py <reference checkout>  (or set PIPPIN_REFERENCE)")
OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "reference_kats.json")


def read(rel):
    with open(os.path.join(REF, rel)) as fh:
        return fh.read()


def line_of(text, needle):
    return text[: text.index(needle)].count("\n") + 1


def main():
    kats = {}
    newton = read("crates/pippin/src/newton.rs")
    m = re.search(r"let s = \[([^\]]+)\];", newton[newton.index("fn impedance_curve"):])
    solimp = [float(x) for x in m.group(1).split(",")]
    cases = re.findall(r"impedance\(&s, ([0-9.e-]+)\) - ([0-9.e-]+)\)\.abs\(\) < ([0-9.e-]+)",
                       newton[newton.index("fn impedance_curve"):])
    kats["impedance"] = {
        "source": f"crates/pippin/src/newton.rs:{line_of(newton, 'fn impedance_curve')}",
        "solimp": solimp,
        "cases": [{"pos": float(p), "expected": float(e), "tol": float(t)} for p, e, t in cases],
    }

    math_rs = read("crates/pippin/src/math.rs")
    blk = math_rs[math_rs.index("fn block_cholesky_matches_dense_on_block_diagonal"):]
    diag = re.search(r"if i == j \{ ([0-9.]+) \+ i as Real \} else \{ ([0-9.]+) \+ ([0-9.]+) \* \(i \+ j\)", blk)
    tol = re.search(r"\(x1\[i\] - x2\[i\]\)\.abs\(\) < ([0-9.e-]+)", blk)
    kats["block_cholesky"] = {
        "source": f"crates/pippin/src/math.rs:{line_of(math_rs, 'fn block_cholesky_matches_dense_on_block_diagonal')}",
        "n": 5, "blocks": [[0, 2], [2, 5]],
        "diag_base": float(diag.group(1)), "off_base": float(diag.group(2)), "off_step": float(diag.group(3)),
        "rhs": "1 + i", "tol": float(tol.group(1)),
    }
    cs = math_rs[math_rs.index("fn cholesky_solves"):]
    a = re.search(r"let mut a = vec!\[([^\]]+)\];", cs)
    x = re.search(r"let mut x = vec!\[([^\]]+)\];", cs)
    t = re.search(r"\]\[i\]\)\.abs\(\) < ([0-9.e-]+)", cs)
    kats["cholesky_solve"] = {
        "source": f"crates/pippin/src/math.rs:{line_of(math_rs, 'fn cholesky_solves')}",
        "a": [float(v) for v in a.group(1).split(",")], "b": [float(v) for v in x.group(1).split(",")],
        "tol": float(t.group(1)),
    }
    qr = math_rs[math_rs.index("fn quat_mat_roundtrip"):]
    q = re.search(r"from_axis_angle\(Vec3::new\(([^)]+)\), ([0-9.]+)\)", qr)
    t = re.search(r"\.abs\(\) < ([0-9.e-]+)", qr)
    kats["quat_roundtrip"] = {
        "source": f"crates/pippin/src/math.rs:{line_of(math_rs, 'fn quat_mat_roundtrip')}",
        "axis": [float(v) for v in q.group(1).split(",")], "angle": float(q.group(2)), "tol": float(t.group(1)),
    }

    simd = read("crates/pippin/src/simd.rs")
    ds = simd[simd.index("fn dot_matches_scalar"):]
    rng = re.search(r"for n in 0\.\.(\d+)", ds)
    fa = re.search(r"\(i as Real \* ([0-9.]+)\)\.sin\(\)", ds)
    fb = re.search(r"\(i as Real \* ([0-9.]+)\)\.cos\(\)", ds)
    t = re.search(r"\.abs\(\) < ([0-9.e-]+)", ds)
    kats["dot"] = {
        "source": f"crates/pippin/src/simd.rs:{line_of(simd, 'fn dot_matches_scalar')}",
        "n_max": int(rng.group(1)), "a_sin_step": float(fa.group(1)), "b_cos_step": float(fb.group(1)),
        "tol": float(t.group(1)),
    }

    mesh = read("crates/pippin/src/mesh.rs")
    cm = mesh[mesh.index("fn cube_mass_properties_are_exact"):]
    h = re.search(r"let h = ([0-9.]+);", cm)
    off = re.search(r"let offset = Vec3::new\(([^)]+)\);", cm)
    t = re.search(r"\(vol - side\.powi\(3\)\)\.abs\(\) < ([0-9.e-]+)", cm)
    kats["cube_mass"] = {
        "source": f"crates/pippin/src/mesh.rs:{line_of(mesh, 'fn cube_mass_properties_are_exact')}",
        "half": float(h.group(1)), "offset": [float(v) for v in off.group(1).split(",")], "tol": float(t.group(1)),
    }
    with open(OUT, "w") as fh:
        json.dump(kats, fh, indent=1)
    print("wrote", OUT)


if __name__ == "__main__":
    main()
