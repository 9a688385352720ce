"""CPU oracle (test infrastructure only): FP64 numpy restatement of the reference
algorithms for the KRFFT / SCFT-diffusion hot path.  Imported only by tests/,
__graft_entry__.smoke() and bench.py's CPU-baseline leg."""
