"""CPU oracle of the HOPS trajectory hot path -- test infrastructure only.

Used by tests/, __graft_entry__.smoke() and the CPU-baseline leg of bench.py
to check and time against; the product package never imports it."""
