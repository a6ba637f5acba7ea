"""Generate tests/golden/reference_kats.json from the reference's own code.

Runs oracle/_ref/ref_kat (built by `make -C oracle ref` from the reference's
GPU_MPM/SPGridMask.cpp, Materials.cpp and the header-only SVD QRSVD.hpp /
givens.hpp) on seeded inputs and records inputs and outputs as hex floats.
Needs the reference sources at build time only; the fixture is committed and
the tests read the fixture.

    python tests/golden/make_golden.py
"""
from __future__ import annotations

import hashlib
import json
import subprocess
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
REF = ROOT / "oracle" / "_ref" / "ref_kat"
OUT = Path(__file__).resolve().parent / "reference_kats.json"


def run(mode: str, stdin: str) -> list[str]:
    r = subprocess.run([str(REF), mode], input=stdin, capture_output=True, text=True, check=True)
    return r.stdout.strip().splitlines()


def svd_inputs(rng: np.random.Generator) -> list[np.ndarray]:
    mats = []
    for t in range(400):
        kind = t % 8
        if kind == 0:
            A = np.eye(3) + 0.05 * rng.standard_normal((3, 3))        # deformation gradients near I
        elif kind == 1:
            A = rng.standard_normal((3, 3))                           # general
        elif kind == 2:
            A = np.diag(rng.uniform(0.3, 3.0, 3))                     # already diagonal
        elif kind == 3:
            A = rng.standard_normal((3, 3))
            A[2] = 0.5 * A[0] + 0.25 * A[1]                           # rank 2
        elif kind == 4:
            Q, _ = np.linalg.qr(rng.standard_normal((3, 3)))
            A = Q @ np.diag([1.0, 1.0, 1e-4]) @ Q.T                   # ill conditioned
        elif kind == 5:
            Q, _ = np.linalg.qr(rng.standard_normal((3, 3)))
            A = Q                                                     # orthogonal (det +-1)
        elif kind == 6:
            A = np.eye(3) + 0.3 * rng.standard_normal((3, 3))
            A[:, 0] *= -1.0                                           # inverted
        else:
            A = np.diag([1.0, 1.0, 1.0]) + 1e-7 * rng.standard_normal((3, 3))  # repeated singular values
        mats.append(A)
    mats.append(np.eye(3))
    mats.append(np.zeros((3, 3)))
    return mats


GOLDEN = Path(__file__).resolve().parent
TUBE = Path("/root/reference/Assets/sample/tube_10.obj")
SDF_CENTER, SDF_RES = (128, 64, 128), (8, 8, 8)


def write_sampler_inputs() -> None:
    """Small committed inputs for the reference's samplers: a sphere level set
    in the reference's SDF text format, and an OBJ with face and normal
    records around its vertices."""
    n = 16
    g = np.arange(n, dtype=np.float64)
    i, j, k = np.meshgrid(g, g, g, indexing="ij")
    phi = np.sqrt((i - 7.3) ** 2 + (j - 7.8) ** 2 + (k - 8.1) ** 2) - 5.2
    vals = phi.transpose(2, 1, 0).ravel()  # i fastest
    lines = [f"{n} {n} {n}", "-0.5 -0.5 -0.5", "0.0625"] + [repr(float(v)) for v in vals]
    (GOLDEN / "sample_sphere.sdf").write_text("\n".join(lines) + "\n")
    rng = np.random.default_rng(5)
    v = rng.uniform(0.0, 1.0, (120, 3)).tolist()
    recs = [f"v {a!r} {b!r} {c!r}" for a, b, c in v[:100]]
    recs += ["f 1 2 3", "f 4 5 6"] + [f"v {a!r} {b!r} {c!r}" for a, b, c in v[100:110]]
    recs += ["vn 0 1 0"] + [f"v {a!r} {b!r} {c!r}" for a, b, c in v[110:]]
    (GOLDEN / "sample_records.obj").write_text("\n".join(recs) + "\n")


def sampler_record(args: list[str]) -> dict:
    r = subprocess.run([str(REF), *args], capture_output=True, text=True, check=True)
    lines = r.stdout.splitlines()
    at = next(i for i, l in enumerate(lines) if l.startswith("COUNT"))
    n = int(lines[at].split()[1])
    pts = np.array([[float.fromhex(x) for x in l.split()] for l in lines[at + 1:at + 1 + n]], dtype=np.float64)
    pts = pts.reshape(-1, 3)
    return {"count": n, "sha1": hashlib.sha1(pts.tobytes()).hexdigest(),
            "first": [x.hex() for x in pts[0]] if n else [], "last": [x.hex() for x in pts[-1]] if n else []}


def sampler_kats() -> dict:
    write_sampler_inputs()
    out = {"sample_records_obj": sampler_record(["obj", str(GOLDEN / "sample_records.obj")]),
           "sample_cube": sampler_record(["cube"]),
           "sample_sdf": dict(center=SDF_CENTER, res=SDF_RES,
                              **sampler_record(["sdf", str(GOLDEN / "sample_sphere.sdf"),
                                                *map(str, SDF_CENTER), *map(str, SDF_RES)]))}
    if TUBE.exists():
        out["sample_tube_10_obj"] = sampler_record(["obj", str(TUBE)])
    return out


def main() -> None:
    if not REF.exists():
        subprocess.run(["make", "-C", str(ROOT / "oracle"), "ref"], check=True)
    out: dict = {"generator": "tests/golden/make_golden.py", "source": "oracle/_ref/ref_kat (reference code)"}
    masks = [l for l in run("masks", "") if l.startswith("MASKS")][0].split()[1:]
    out["masks"] = masks
    rng = np.random.default_rng(20201120)
    pts = [(3, 1, 2), (8, 8, 13), (13, 15, 24), (18, 22, 35), (0, 0, 0), (255, 255, 255), (4, 0, 0), (0, 4, 0),
           (0, 0, 4)] + [tuple(int(v) for v in rng.integers(0, 1020, 3)) for _ in range(200)]
    lines = run("offsets", "\n".join(f"{i} {j} {k}" for i, j, k in pts) + "\n")
    out["offsets"] = [[int(a), int(b), int(c), d] for a, b, c, d in (l.split()[1:] for l in lines if l.startswith("OFFSET"))]
    mats_in = [(1e5, 0.3, 1000.0, 1.0), (2e2, 0.4, 3.0, 1.0), (5e4, 0.25, 1000.0, 1.0), (5e5, 0.3, 1000.0, 1.0),
               (3000.0, 0.4, 24.0, 1.0)]
    lines = run("material", "\n".join(" ".join(repr(x) for x in m) for m in mats_in) + "\n")
    out["materials"] = [{"E": m[0], "nu": m[1], "lambda": l.split()[1], "mu": l.split()[2], "kappa": l.split()[3],
                         "M": l.split()[4]} for m, l in zip(mats_in, lines)]
    svd_in = svd_inputs(rng)
    lines = run("svd", "\n".join(" ".join(float(x).hex() for x in A.ravel()) for A in svd_in) + "\n")
    out["svd"] = [{"F": [float(x).hex() for x in A.ravel()], "USV": l.split()[1:]} for A, l in zip(svd_in, lines)]
    out.update(sampler_kats())
    OUT.write_text(json.dumps(out, separators=(",", ":")))
    print(f"wrote {OUT} ({len(out['svd'])} SVD cases, {len(out['offsets'])} offsets)")


if __name__ == "__main__":
    main()
