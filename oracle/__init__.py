"""CPU oracle (test infrastructure): numpy restatements of the reference's
RF demodulator and time-base corrector, used only as the checker of the
CUDA path by tests/, __graft_entry__.smoke() and bench.py's CPU baseline."""
