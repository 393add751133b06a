"""CPU oracle for the XPRecon hot path: test infrastructure only (never imported by the product)."""
