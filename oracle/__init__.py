"""CPU restatement of RadiativeViewFactor.jl's assembly path (test infrastructure only)."""
