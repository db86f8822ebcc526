"""Oracle (test infrastructure): CPU restatement of the reference stepper. Not product code."""
