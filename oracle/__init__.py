"""CPU oracle (test infrastructure only): an OpenMP transcription of the
reference kernel logic, used by tests/, __graft_entry__.smoke() and bench.py's
CPU-baseline leg as the checker. The product never imports this package."""
