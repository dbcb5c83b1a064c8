"""fluidmaxxer_b200 -- FluidMaxxer's coupled lattice-Boltzmann time step on B200.

D3Q19 BGK / porous-BGK Navier-Stokes, D3Q7 BGK advection-diffusion driven by
the NS velocity, and linear / Langmuir LDF adsorption, as fused sm_100a CUDA
kernels behind the C ABI of ``include/fm.h`` (``libfm.so``).

Modules:
    _abi      ctypes declarations of the C ABI (fails loudly without libfm.so)
    lattice   CoupledLattice host binding and the main.cpp-style set-up
    problems  workload descriptions and seeded geometries
    synth     seeded geometry generators (host)
    build     in-tree build of the native libraries
"""

__all__ = ["lattice", "problems", "synth", "build"]
__version__ = "0.1.0"
