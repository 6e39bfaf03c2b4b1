"""CPU oracle for the tet-DG RHS hot path: test infrastructure only (never imported by the product)."""
