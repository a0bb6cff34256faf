"""CPU oracle (test infrastructure): an FP64 C restatement of the reference
routines on the solvent hot path, used only by tests, smoke() and the CPU
baseline of bench.py."""
