"""CPU oracle for the dense statevector path — test infrastructure only."""
