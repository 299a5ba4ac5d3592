"""CPU oracle of the warpSPH hot path -- test infrastructure, never imported by warpsph_b200."""
