"""TEST INFRASTRUCTURE ONLY: the CPU oracle (C++ restatement of the reference
engine) and its ctypes wrapper.  Imported by tests/, the smoke check and
bench.py's CPU-baseline leg only."""
