"""Golden vectors from the reference itself: runs the reference's own CUDA
kernels (oracle/_ref/libostc_ref_cuda.so, built from the reference sources
by oracle/build_ref.sh) on small seeded cases and stores what they produce,
so that the CPU oracle can be pinned without a GPU (tests/test_golden_cpu.py).

Needs a GPU and the reference build; writes one compressed .npz per case:

    python tests/golden/make_golden.py --out tests/golden

Each file holds, per block b: the SHA-256 of the block's inputs (bv, sv,
jac, metric as built by the case builder, to detect builder drift), the
interior RHS dq after initialisation (`dq_b`), and after the case's steps
the interior bv / sv (species and SST k, omega: `bv_b`, `sv_b`) plus the residual history `res` and,
for RK3, the dt history `dt`; `reduction_ok` says whether the reference's
block reductions are well defined at these sizes (they are for every case
here)."""
import argparse
import hashlib
import sys
from pathlib import Path

import numpy as np

REPO = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(REPO / "openstc-dev_b200"))
sys.path.insert(0, str(REPO / "tests"))

import ostc  # noqa: E402


def _no_periodic(c):
    for f in c.faces:
        if f.type_label == ostc.BC_PERIODIC:
            f.type_label = ostc.BC_OUTFLOW
    return c


def _mixing(recon=2, inv=3):
    c = _no_periodic(ostc.case_mixing_layer(12, 10, 6, full_host=True))
    c.scheme.reconstruction, c.scheme.inviscid_scheme = recon, inv
    return c


def _vortex(recon, inv):
    return ostc.case_vortex(16, 12, 6, k_bc="symmetry", reconstruction=recon, inviscid_scheme=inv)


def _sst_air():
    """one walled SST block (case_uneven_blocks); the far field becomes outflow because the
    reference's air + SST far field reads unset boundary scalars (quirk A20)"""
    c = ostc.case_uneven_blocks(layout=[((0, 0, 0), (18, 14, 6))], rans_model=2)
    for f in c.faces:
        if f.type_label == ostc.BC_FARFIELD:
            f.type_label = ostc.BC_OUTFLOW
    return c


def _sst_h2air():
    """the reacting mixing layer with SST and an isothermal wall at j = 0 (Driver<FR, SST>)"""
    return _no_periodic(ostc.case_mixing_layer(12, 11, 6, full_host=True, rans_model=2, wall=True))


# name -> (builder, mode, steps); mode "rk3" or "steady"
CASES = {
    "vortex_aweno": (lambda: _vortex(4, 2), "rk3", 5),
    "vortex_roe_muscl": (lambda: _vortex(2, 2), "rk3", 5),
    "vortex_hllc_nnd2": (lambda: _vortex(3, 4), "rk3", 5),
    "vortex_lf_first": (lambda: _vortex(1, 1), "rk3", 5),
    "mixing_ausm_muscl": (lambda: _mixing(2, 3), "rk3", 3),
    "mixing_roe_muscl": (lambda: _mixing(2, 2), "rk3", 3),
    "bc_wall_farfield": (lambda: ostc.case_bc_box("wall_farfield", 20, 16, 6), "rk3", 4),
    "bc_subsonic": (lambda: ostc.case_bc_box("subsonic", 20, 16, 6), "rk3", 4),
    "multiblock_aweno": (lambda: ostc.case_multiblock((9, 8), (7, 9), 6), "rk3", 3),
    "premixed_steady_epi": (lambda: ostc.make_steady(ostc.case_premixed_box(12, 10, 6), 0, 1), "steady", 4),
    "premixed_dplur_epi": (lambda: ostc.make_steady(ostc.case_premixed_box(12, 10, 6), 1, 1), "steady", 4),
    "premixed_dplur_da": (lambda: ostc.make_steady(ostc.case_premixed_box(12, 10, 6), 1, 2), "steady", 4),
    "wall_dplur": (lambda: ostc.make_steady(ostc.case_bc_box("wall_farfield", 20, 16, 6), 1), "steady", 4),
    "sst_air_hllc": (_sst_air, "rk3", 4),
    "sst_air_dplur": (lambda: ostc.make_steady(_sst_air(), 1), "steady", 4),
    "sst_h2air_wall": (_sst_h2air, "rk3", 3),
    "sst_h2air_dplur_epi": (lambda: ostc.make_steady(_sst_h2air(), 1, 1), "steady", 3),
    "planar_roe_muscl": (lambda: ostc.case_vortex(25, 21, 1, reconstruction=2, inviscid_scheme=2), "rk3", 5),
    "planar_wall_dplur": (lambda: ostc.make_steady(ostc.case_bc_box("wall_farfield", 25, 21, 1), 1), "steady", 4),
}


def input_digest(block):
    h = hashlib.sha256()
    for n in ("bv", "sv", "jac", "metric"):
        v = block.arrays.get(n)
        if v is not None and v.size:
            h.update(np.ascontiguousarray(v).view(np.uint8).tobytes())
    return h.hexdigest()


def reduction_well_defined(cells):
    # block_reduce_{min,sum} read an unwritten shared slot when the valid
    # thread count of the last block of a pass is a multiple of 32 below 128
    nb = (cells + 127) // 128
    v1, v2 = cells - (nb - 1) * 128, nb
    return all(v == 128 or v % 32 for v in (v1, v2))


def interior(a, g):
    """interior of a ghosted array with a leading variable axis"""
    if g == 0:
        return np.ascontiguousarray(a)
    return np.ascontiguousarray(a[:, g:a.shape[1] - g, g:a.shape[2] - g, g:a.shape[3] - g])


def main():
    import ref_bind

    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=str(REPO / "tests" / "golden"))
    a = ap.parse_args()
    out = Path(a.out)
    out.mkdir(parents=True, exist_ok=True)
    for name, (build, mode, steps) in CASES.items():
        case = build()
        data = {"mode": np.array(mode), "steps": np.array(steps),
                "reduction_ok": np.array(all(reduction_well_defined(b.mx * b.my * b.mz) for b in case.blocks))}
        r = ref_bind.RefCudaRun(case)
        r.initialize()
        r.compute_rhs()
        for b, blk in enumerate(case.blocks):
            data["digest_%d" % b] = np.array(input_digest(blk))
            data["dq_%d" % b] = interior(r.download("dq", b), blk.dq_ngg)
        r2 = ref_bind.RefCudaRun(case)
        r2.initialize()
        if mode == "rk3":
            res, dts = r2.rk3_steps(steps)
            data["dt"] = dts
        else:
            res = r2.steady_steps(steps)
        data["res"] = res
        for b, blk in enumerate(case.blocks):
            data["bv_%d" % b] = interior(r2.download("bv", b), blk.ngg)
            if blk.n_spec + blk.n_turb:
                data["sv_%d" % b] = interior(r2.download("sv", b), blk.ngg)
        np.savez_compressed(out / ("%s.npz" % name), **data)
        print("wrote", name, sum(v.nbytes for v in data.values()))


if __name__ == "__main__":
    main()
