"""Power-network callers of the device solve: a PyPSA CSV network reader and
the dispatch LOPF builder (the LP family the benchmark workloads come from)."""
