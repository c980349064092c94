"""ORACLE TEST INFRASTRUCTURE — CPU restatements of the reference's hot path
and the reference's own shader compiled for the host.  Used only by tests/,
the smoke check and bench.py's CPU-baseline leg; never by the product."""
