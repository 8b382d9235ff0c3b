"""CPU oracle of the dictionary-indexing path. Test infrastructure only: used
by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg, never by
the ebsdtorch_b200 product path."""
