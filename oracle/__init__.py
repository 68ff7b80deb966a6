"""CPU oracle for the Wick (H, S) path: test infrastructure only (see each module header)."""
