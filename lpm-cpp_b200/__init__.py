"""B200-native implicit quasi-static step of the nonlocal lattice particle method (LPM).

The CUDA kernels and the C ABI live in ``csrc/`` and build into ``liblpmgpu.so`` beside this
file (``build.py``); ``lpm.py`` is the host-side mirror of the LPM-CPP interface over that ABI.
The directory name is not a Python identifier, so import it with
``importlib.import_module("lpm-cpp_b200.lpm")``.
"""
