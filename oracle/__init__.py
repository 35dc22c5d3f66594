"""CPU oracle of the pusher path -- test infrastructure only (tests/,
__graft_entry__.smoke() and bench.py's CPU-baseline leg use it as the
checker; the product never imports it)."""
