"""CPU oracle of the FerroX coupled time step -- test infrastructure only.

Used by tests/, ``__graft_entry__.smoke()`` and bench.py's cpu_baseline leg as
the checker; the ferrox_b200 product never imports it.
"""
