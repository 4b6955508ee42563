"""B200-native Lanczos hot path of the NuShellX shell-model code.

* ``nushellx_b200.nsx``   -- Python binding of libnsx.so (CUDA H.v, thick-restart
                             Lanczos, C ABI of include/nsx.h)
* ``nushellx_b200.gen``   -- synthetic producer of the reference's input files
                             (.tri/.trd densities, .oph, .mat/.sgt, .spe)
* ``nushellx_b200.build`` -- nvcc build of libnsx.so for sm_100a
"""
