"""FP64 CPU oracle (test infrastructure only; the product never imports this package)."""
