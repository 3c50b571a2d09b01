"""Test infrastructure: the CPU f64 oracle.  Never imported by the engine."""
