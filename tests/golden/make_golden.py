"""Regenerate the golden fixtures of tests/golden from the reference (hsolve) checkout.

Run in a container that has a checkout of the reference; its path REF is a required argument. The
fixtures it writes are committed, so the tests never read the reference at run time:

    python tests/golden/make_golden.py REF

Fixtures
* yee_spectra.npz   exact discrete Yee spectra from the reference's own closed form
                    (tools/gen/yee.py:231 exact_eigenvalues) for several boxes: pins oracle/yee_exact.py
* yee_matrices.npz  small Yee pencils assembled by the reference generator (tools/gen/yee.py:182
                    assemble, :211 standard_form): pins hsolve_b200/gen/yee.py
* examples.json     the reference's example cases (examples/cases/*/{meta,config}.json): target,
                    inertia of A, a digest of the stored A, and the reference eigenvalues that the
                    target needs (examples/refs/*/eigenvalues.npy), for cases our generator rebuilds
* near_singular.npz the near-singular-shift example (prescribed-spectrum matrix, n = 2000) with its
                    exact spectrum: the null-pivot / singular-shift known answers
* waveguide.npz     the GHIEP waveguide-50ghz example (A, B indefinite) with its dense spectrum
"""
from __future__ import annotations

import hashlib
import json
import sys
from pathlib import Path

import numpy as np
import scipy.sparse as sp

HERE = Path(__file__).resolve().parent


def digest(m) -> dict:
    m = sp.csr_matrix(m)
    m.sort_indices()
    return {"n": int(m.shape[0]), "nnz": int(m.nnz), "abs_sum": float(np.abs(m.data).sum()),
            "trace": float(m.diagonal().real.sum()),
            "pattern_sha256": hashlib.sha256(np.ascontiguousarray(m.indices.astype(np.int64)).tobytes()
                                             + np.ascontiguousarray(m.indptr.astype(np.int64)).tobytes()).hexdigest()}


def main(ref: str) -> None:
    sys.path.insert(0, ref)
    from tools.gen import yee as R  # the reference generator

    boxes = {
        "pec_4x3x5": R.YeeGrid((4, 3, 5)),
        "pec_box_5x4x3": R.YeeGrid((5, 4, 3), (1.0, 0.7, 0.45)),
        "pec_cube16": R.YeeGrid((16, 16, 16)),
        "pec_cube20": R.YeeGrid((20, 20, 20)),
        "pec_box1e5": R.YeeGrid((44, 34, 26), (1.0, 0.75, 0.55)),
        "bloch_4x3x3": R.YeeGrid((4, 3, 3), (1.0, 0.9, 0.8), "bloch", (0.3 * np.pi, 0.2 * np.pi, 0.1 * np.pi)),
        "bloch_gamma_3x3x3": R.YeeGrid((3, 3, 3), (1.0, 1.0, 1.0), "bloch", (0.0, 0.0, 0.0)),
    }
    spectra = {}
    for name, g in boxes.items():
        spectra[name] = R.exact_eigenvalues(g)
        spectra[name + "__params"] = np.array([*g.cells, *g.lengths, *g.phases, g.boundary == "pec"], dtype=float)
    np.savez_compressed(HERE / "yee_spectra.npz", **spectra)

    mats = {}
    for name in ("pec_4x3x5", "pec_box_5x4x3", "bloch_4x3x3"):
        g = boxes[name]
        a, b = R.assemble(g)
        s = R.standard_form(a, b)
        for tag, m in (("A", a), ("B", b), ("S", s)):
            m = sp.csr_matrix(m)
            m.sort_indices()
            mats[f"{name}__{tag}_data"] = m.data
            mats[f"{name}__{tag}_indices"] = m.indices.astype(np.int32)
            mats[f"{name}__{tag}_indptr"] = m.indptr.astype(np.int64)
    # one inhomogeneous (photonic sphere) pencil
    g = R.YeeGrid((4, 4, 4), (1.0, 1.0, 1.0), "bloch", (0.4 * np.pi, 0.25 * np.pi, 0.1 * np.pi))
    eps = R.photonic_permittivity(g, "spheres", 0.25, 12.0)
    a, b = R.assemble(g, eps=eps)
    for tag, m in (("A", a), ("B", b)):
        m = sp.csr_matrix(m)
        m.sort_indices()
        mats[f"sphere_4x4x4__{tag}_data"] = m.data
        mats[f"sphere_4x4x4__{tag}_indices"] = m.indices.astype(np.int32)
        mats[f"sphere_4x4x4__{tag}_indptr"] = m.indptr.astype(np.int64)
    mats["sphere_4x4x4__eps"] = eps
    np.savez_compressed(HERE / "yee_matrices.npz", **mats)

    ex_root = Path(ref) / "examples"
    examples = {}
    for case_dir in sorted((ex_root / "cases").iterdir()):
        meta = json.loads((case_dir / "meta.json").read_text())
        cfg = json.loads((case_dir / "config.json").read_text())
        w = np.load(ex_root / "refs" / case_dir.name / "eigenvalues.npy")
        a = sp.load_npz(case_dir / "A.npz")
        entry = {"meta": meta, "config": cfg, "A_digest": digest(a)}
        if (case_dir / "B.npz").exists():
            entry["B_digest"] = digest(sp.load_npz(case_dir / "B.npz"))
        tgt = cfg["target"]
        wr = np.sort(np.real(w))
        if tgt["mode"] == "nearest":
            order = np.argsort(np.abs(wr - tgt["sigma"]), kind="stable")
            entry["ref_nearest"] = [float(x) for x in wr[order[: tgt["k"] + 8]]]
        else:
            inside = wr[(wr >= tgt["lower"]) & (wr <= tgt["upper"])]
            entry["ref_interval"] = [float(x) for x in inside]
            entry["ref_below_lower"] = int(np.searchsorted(wr, tgt["lower"], side="left"))
            entry["ref_below_upper_excl"] = int(np.searchsorted(wr, tgt["upper"], side="right"))
        examples[case_dir.name] = entry
    (HERE / "examples.json").write_text(json.dumps(examples, indent=1) + "\n")

    a = sp.csr_matrix(sp.load_npz(ex_root / "cases" / "near-singular-shift" / "A.npz"))
    a.sort_indices()
    w = np.load(ex_root / "refs" / "near-singular-shift" / "eigenvalues.npy")
    np.savez_compressed(HERE / "near_singular.npz", data=a.data, indices=a.indices.astype(np.int32),
                        indptr=a.indptr.astype(np.int64), eigenvalues=np.sort(np.real(w)))

    wa = sp.csr_matrix(sp.load_npz(ex_root / "cases" / "waveguide-50ghz" / "A.npz"))
    wb = sp.csr_matrix(sp.load_npz(ex_root / "cases" / "waveguide-50ghz" / "B.npz"))
    wa.sort_indices(), wb.sort_indices()
    w = np.load(ex_root / "refs" / "waveguide-50ghz" / "eigenvalues.npy")
    np.savez_compressed(HERE / "waveguide.npz", A_data=wa.data, A_indices=wa.indices.astype(np.int32),
                        A_indptr=wa.indptr.astype(np.int64), B_data=wb.data,
                        B_indices=wb.indices.astype(np.int32), B_indptr=wb.indptr.astype(np.int64),
                        eigenvalues=w)
    print("wrote", sorted(p.name for p in HERE.iterdir()))


if __name__ == "__main__":
    if len(sys.argv) != 2:
        raise SystemExit("usage: python tests/golden/make_golden.py REF  (path of the reference checkout)")
    main(sys.argv[1])
