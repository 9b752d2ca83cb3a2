"""CPU oracle for the Barnes-Hut evolution path (test infrastructure only)."""
