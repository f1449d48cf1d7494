"""physik_b200 -- PhysiK's implicit soft-body step on B200 (sm_100a).

The product is the pair of in-tree shared libraries under ``physik_b200/lib``:
``libpkcuda.so`` (CUDA kernels + the thin device C ABI of ``include/pkcuda.h``) and
``libphysik_b200.so`` (the C++ host layer that mirrors PhysiK's World / component /
solver API and exports the drop-in ``PHYSIK_*`` C ABI of ``include/physik_b200.h``).
This Python package only loads them (``_lib``), wraps the C ABI for tests and the
benchmark (``world``) and generates the synthetic workloads (``meshes``).
"""
__all__ = ["meshes"]
