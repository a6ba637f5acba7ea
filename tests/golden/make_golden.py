"""Generate the known-answer fixtures from the reference's own code.

tests/golden/reference_kats.json: oracle/_ref/ref_kat (built by
`make -C oracle ref` from the reference's GPU_MPM/SPGridMask.cpp,
Materials.cpp, LoadSample.cpp and the header-only SVD QRSVD.hpp / givens.hpp)
on seeded inputs, inputs and outputs as hex floats.

tests/golden/reference_kernel_kats.json: oracle/_ref/ref_kernels, the
reference's per-thread kernels applyVonMises + computePhase_field_vol,
undateGrid_kernal + collideWithGround / PullGrid_kernal, and cal_cellId +
calcIndex run serially on the host, on seeded cases chosen to reach every
branch (elastic, yielding, the alpha, dlambda and strain caps, J < 1 and
J >= 1, softening, the psi cap, the hydrostatic trial state, inverted F;
tagged and untouched nodes, a non-finite force, walls on every face, the two
moving spheres; cells on rounding boundaries and outside the domain).  Arrays
are stored as base64 of zlib-compressed little-endian float64 (bit exact).

Needs the reference sources at build time only (their root in the environment
variable GMPM_REFERENCE_DIR); the fixtures are committed and the tests read
the fixtures.

    GMPM_REFERENCE_DIR=<reference root> python tests/golden/make_golden.py
"""
from __future__ import annotations

import base64
import hashlib
import json
import os
import subprocess
import zlib
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
REF = ROOT / "oracle" / "_ref" / "ref_kat"
REF_KERNELS = ROOT / "oracle" / "_ref" / "ref_kernels"
OUT = Path(__file__).resolve().parent / "reference_kats.json"
OUT_KERNELS = Path(__file__).resolve().parent / "reference_kernel_kats.json"
REFERENCE_DIR = os.environ.get("GMPM_REFERENCE_DIR", "")


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
TUBE = Path(REFERENCE_DIR) / "Assets" / "sample" / "tube_10.obj"
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
    if REFERENCE_DIR and TUBE.exists():
        out["sample_tube_10_obj"] = sampler_record(["obj", str(TUBE)])
    return out


def pack(a: np.ndarray) -> dict:
    a = np.ascontiguousarray(a, dtype="<f8")
    return {"shape": list(a.shape), "zb64": base64.b64encode(zlib.compress(a.tobytes(), 9)).decode()}


def run_kernels(mode: str, stdin: str, tag: str) -> np.ndarray:
    r = subprocess.run([str(REF_KERNELS), mode], input=stdin, capture_output=True, text=True, check=True)
    rows = [l.split()[1:] for l in r.stdout.splitlines() if l.startswith(tag)]
    return np.array([[float.fromhex(x) for x in row] for row in rows], dtype=np.float64)


def hexline(vals) -> str:
    return " ".join(float(v).hex() for v in vals)


# Materials (E, nu) and grid spacings of the constitutive cases: the notched
# bar's material, the reference's own scene material (Simulator.cpp:114-116)
# and the extremes of the plates' drawn stiffness.
VM_MATERIALS = [(1e5, 0.3), (2e2, 0.4), (5e4, 0.25), (5e5, 0.3)]
VM_DX = [1.0 / 256, 1.0 / 128]


def vm_cases(rng: np.random.Generator) -> tuple[np.ndarray, list[str]]:
    """Rows: E nu dx V0 F(9, column-major) g alpha c psi_max; and a label each."""
    rows, labels = [], []

    def add(label, F, g=1.0, alpha=0.0, c=1.0, psi=0.0, mat=None, dx=None):
        E, nu = mat if mat is not None else VM_MATERIALS[len(rows) % len(VM_MATERIALS)]
        h = dx if dx is not None else VM_DX[(len(rows) // 4) % 2]
        rows.append([E, nu, h, h ** 3 / 8, *np.asarray(F, dtype=np.float64).T.ravel(), g, alpha, c, psi])
        labels.append(label)

    def rot():
        Q, _ = np.linalg.qr(rng.standard_normal((3, 3)))
        return Q if np.linalg.det(Q) > 0 else -Q

    for _ in range(24):  # elastic: strains far below 800 Pa / E
        add("elastic", np.eye(3) + 1e-6 * rng.standard_normal((3, 3)), mat=(1e5, 0.3))
    for _ in range(8):
        add("elastic", np.eye(3) + 1e-3 * rng.standard_normal((3, 3)), mat=(2e2, 0.4))
    for _ in range(40):  # yielding, J on both sides of 1
        add("yield", np.eye(3) + 0.05 * rng.standard_normal((3, 3)), alpha=float(rng.uniform(0, 0.5)),
            c=float(rng.uniform(0.2, 1.0)), g=float(rng.uniform(0.05, 1.0)), psi=float(rng.uniform(0, 50)))
    for _ in range(16):  # compression J < 1
        add("compress", (0.9 + 0.02 * rng.standard_normal()) * rot() @ np.diag(rng.uniform(0.93, 1.0, 3)),
            alpha=float(rng.uniform(0, 0.3)))
    for _ in range(16):  # expansion J > 1
        add("expand", rot() @ np.diag(rng.uniform(1.0, 1.08, 3)) @ rot(), alpha=float(rng.uniform(0, 0.3)))
    for a in (0.985, 0.995, 0.9999, 1.0, 1.2):  # alpha reaching, at or above its cap
        for _ in range(3):
            add("alpha_cap", np.eye(3) + 0.05 * rng.standard_normal((3, 3)), alpha=a)
    for d in (1e-7, 1e-9, 1e-11):  # isochoric stretch with a tiny positive trace: dlambda above 100
        for _ in range(3):
            e = float(rng.uniform(0.02, 0.2))
            eps = np.array([e, -e / 2, -e / 2 + d])
            Q = rot()
            add("dlambda_cap", Q @ np.diag(np.exp(eps)) @ Q.T)
    for s in (25.0, 40.0, 80.0):  # Hencky strain above the clamp of 3
        add("strain_cap", np.diag([s, 1.0, 1.0]))
        add("strain_cap", rot() @ np.diag([s, 0.9, 1.1]) @ rot())
    for p in (0.03, 0.2, 0.6):  # alpha/2 above ps = 0.01: softened G_c
        for _ in range(3):
            add("softening", np.eye(3) + 0.05 * rng.standard_normal((3, 3)), alpha=p,
                psi=float(rng.uniform(0, 200)), c=float(rng.uniform(0, 1)))
    for _ in range(4):  # tensile energy near the psi cap of 1e6
        add("psi_cap", np.diag([2.5, 2.3, 2.7]) @ rot(), psi=float(rng.uniform(9e5, 1.1e6)), mat=(5e5, 0.3))
    for s in (1.001, 1.05, 0.97):  # hydrostatic trial state: zero deviator (reference: NaN when it yields)
        add("hydrostatic", s * np.eye(3))
    for _ in range(4):  # inverted F (det < 0)
        F = np.eye(3) + 0.2 * rng.standard_normal((3, 3))
        F[:, 0] *= -1.0
        add("inverted", F)
    add("identity", np.eye(3))
    return np.array(rows, dtype=np.float64), labels


# Grid cases: nodes of a 256^3 grid (N = 256 in Setting.h); pages along every
# face for the walls, around the two PullGrid spheres, and in the interior.
GRID_PAGES = [(0, 10, 10), (63, 20, 20), (10, 0, 10), (20, 63, 20), (10, 10, 0), (20, 20, 63), (1, 1, 1),
              (62, 62, 62), (32, 19, 16), (44, 19, 16), (32, 19, 48), (44, 19, 45), (32, 31, 14), (30, 30, 30)]


def grid_cases(rng: np.random.Generator) -> np.ndarray:
    rows = []
    for (bx, by, bz) in GRID_PAGES:
        ch = np.zeros((64, 10))
        for node in range(64):
            r = rng.random()
            if r < 0.1:
                continue  # untouched node: tag 0, all channels 0
            m = float(rng.uniform(1e-9, 1e-6))
            v = rng.uniform(-2, 2, 3)
            ch[node, 0] = m
            ch[node, 1:4] = m * v
            ch[node, 4:7] = rng.uniform(-1e-3, 1e-3, 3)
            w = float(rng.uniform(1e-3, 3.0))
            ch[node, 8] = w
            ch[node, 7] = w * float(rng.uniform(0, 1))
            ch[node, 9] = 0.01 * int(rng.integers(1, 27))
            if r > 0.98:
                ch[node, 4 + int(rng.integers(0, 3))] = np.inf  # skipped by the finiteness test
        rows.append([bx, by, bz, *ch.ravel()])
    return np.array(rows, dtype=np.float64)


def cell_cases(rng: np.random.Generator) -> np.ndarray:
    rows = []
    for inv_dx in (256.0, 128.0):
        h = 1.0 / inv_dx
        for _ in range(150):
            rows.append([inv_dx, *rng.uniform(0.5 * h, 1.0 - 3 * h, 3)])
        for _ in range(40):  # on node and half-node boundaries, where truncation decides
            k = rng.integers(1, int(inv_dx) - 3, 3)
            off = rng.choice([0.0, 0.5], 3)
            rows.append([inv_dx, *((k + off) * h)])
        rows.append([inv_dx, 0.5 * h, 0.5 * h, 0.5 * h])   # lowest in-domain base node 0
        rows.append([inv_dx, 0.25 * h, 0.5, 0.5])          # below it: reference forms node -1 (quirk 13)
        rows.append([inv_dx, 0.5, -0.25 * h, 0.5])
    return np.array(rows, dtype=np.float64)


def kernel_kats() -> dict:
    rng = np.random.default_rng(20201121)
    out: dict = {"generator": "tests/golden/make_golden.py",
                 "source": "oracle/_ref/ref_kernels (reference kernels run serially on the host)"}
    vm_in, labels = vm_cases(rng)
    vm_out = run_kernels("vonmises", "\n".join(hexline(r) for r in vm_in) + "\n", "VM")
    assert vm_out.shape == (len(vm_in), 23)
    out["vonmises"] = {"in": pack(vm_in), "out": pack(vm_out), "labels": labels}
    gin = grid_cases(rng)
    grid = {"in": pack(gin), "runs": []}
    for bc, t, dt in ((0, 0.0, 5e-5), (1, 0.0, 1e-4), (2, 0.1, 5e-5), (2, 0.5, 5e-5)):
        head = hexline([dt, t, bc])
        gout = run_kernels("grid", head + "\n" + "\n".join(hexline(r) for r in gin) + "\n", "GRID")
        assert gout.shape == (len(gin), 256)
        grid["runs"].append({"bc": bc, "t": t, "dt": dt, "out": pack(gout)})
    out["grid"] = grid
    cin = cell_cases(rng)
    r = subprocess.run([str(REF_KERNELS), "cell"], input="\n".join(hexline(x) for x in cin) + "\n",
                       capture_output=True, text=True, check=True)
    rows = [l.split()[1:] for l in r.stdout.splitlines() if l.startswith("CELL")]
    out["cell"] = {"in": pack(cin), "offset": [x[0] for x in rows], "node": [[int(v) for v in x[1:]] for x in rows]}
    return out


def main() -> None:
    if not (REF.exists() and REF_KERNELS.exists()):
        if not REFERENCE_DIR:
            raise SystemExit("set GMPM_REFERENCE_DIR to the reference project's root")
        subprocess.run(["make", "-C", str(ROOT / "oracle"), "ref", f"REF={REFERENCE_DIR}"], check=True)
    OUT_KERNELS.write_text(json.dumps(kernel_kats(), separators=(",", ":")))
    print(f"wrote {OUT_KERNELS}")
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
