"""Lattices up to the size limit (19 planes of 32-bit element offsets: at
most 226,050,000 cells).  No oracle finishes at this size, so the check is a
property of the step: a lattice periodic in z whose geometry repeats every P
planes advances exactly as its P-plane tile does, whatever nz is.  Each big
lattice is compared bit for bit, plane by plane of populations, with the
tile; the tile's z = 0 and z = P-1 planes take the neighbour-table pulls of
the y/z faces and the big lattice's matching planes the constant-offset pulls,
so both pull forms meet at every plane boundary of the tile.  The tile itself
is checked against the oracle by the parity tests.

Sizes (512 x 512 x nz): 856 planes (224.4M cells, the last population planes
past 2^31 elements, near the limit); 456 planes (119.5M), the first multiple
of P where the 16-bit step switches to unsigned pull offsets; 448 planes
(117.4M), the last that keeps the signed ones; and 856 planes in the FP16
pair layout (two cells per 32-bit word, the staged kernel)."""
import numpy as np
import pytest

from fluidmaxxer_b200 import lattice, problems, slabs
from fluidmaxxer_b200._abi import check

pytestmark = pytest.mark.gpu

NX, NY, P = 512, 512, 8
STEPS = 6
SIGNED_LIMIT = 2 ** 31           # 18 ns + nx ny + 2 nx + 1 below it: signed offsets


def _problem(nz, solid_tile):
    solid = np.ascontiguousarray(np.tile(solid_tile, (nz // P, 1, 1)).reshape(-1))
    return problems.Problem(nx=NX, ny=NY, nz=nz, solid=solid, periodic=(False, True, True),
                            isotherm="linear", sample_every=0, steps=STEPS, name=f"tiled_{nz}")


def _solid_tile(seed=4242):
    rng = np.random.default_rng(seed)
    t = (rng.random((P, NY, NX)) < 0.15).astype(np.uint8)
    t[:, :, :3] = 0                # inlet rows and the x = 1 cells they read stay fluid
    t[:, :, NX - 3:] = 0           # so do the outlet rows
    return t


def _planes(L, prec, zs):
    import torch

    nbytes = slabs.PLANE_POPULATIONS * NX * NY * slabs.ELEMENT_BYTES[prec]
    out = []
    for z in zs:
        t = torch.empty(nbytes, dtype=torch.uint8, device="cuda")
        check(L._lib.fm_pack_zplane(L.h, int(z), t.data_ptr()))
        out.append(t)
    torch.cuda.synchronize()
    return out


@pytest.mark.parametrize("prec,nz,pair", [("f32", 856, False), ("f16", 856, False), ("f16", 456, False),
                                          ("f16", 448, False), ("f64", 456, False), ("f16", 856, True)])
def test_tiled_lattice_steps_as_its_tile(prec, nz, pair):
    """FP32 and FP64 (reference-order cell update) and FP16 shifted (deviation
    form); FP16 + fixed-point AD is left out because its stochastic rounding is
    keyed on the cell index, which differs between the lattice and its tile."""
    import torch

    n = NX * NY * nz
    wide = 18 * n + NX * NY + 2 * NX + 1 >= SIGNED_LIMIT
    tile = _solid_tile()
    small = lattice.from_problem(_problem(P, tile), prec, probe=False)
    small.set_pair_layout(pair)
    small.step(STEPS)
    ref = _planes(small, prec, range(P))
    small.close()

    big = lattice.from_problem(_problem(nz, tile), prec, probe=False)
    big.set_pair_layout(pair)
    if pair:
        assert big.step_kernel() == "pair-staged"
    else:
        assert big.step_kernel() == ("one-cell-wide" if wide and prec == "f16" else "one-cell")
    big.step(STEPS)
    zs = [0, 1, P - 1, P, P + 1, 2 * P - 1, nz // 2, nz // 2 + 1, nz - P - 1, nz - P, nz - 2, nz - 1]
    got = _planes(big, prec, zs)
    rho = big.reduce()[0]
    big.close()
    lattice.trim_memory()
    torch.cuda.empty_cache()
    for z, g in zip(zs, got):
        r = ref[z % P]
        bad = int((g != r).sum())
        assert bad == 0, (z, bad)
    assert np.isfinite(rho)
