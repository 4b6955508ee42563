"""Test infrastructure: CPU oracles of the Lanczos hot path.

Only tests/, the smoke check of __graft_entry__ and the CPU-baseline leg of
bench.py use this package, and only as the checker -- never as the code under
measurement.  The product path (nushellx_b200/libnsx.so) does not import it.

* mscheme.py  -- independent M-scheme FP64 diagonalisation (pins the generator's
                 phase and normalisation conventions);
* jscheme.py  -- FP64 restatement of the reference's J-scheme H.v reading the
                 reference-format files;
* nsx_ref.c   -- C/OpenMP restatement of the reference's Lanczos (FP32 storage,
                 axpy-form products), the timed host-core baseline.
"""
