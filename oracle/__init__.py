"""CPU restatement of the reference path: test infrastructure only (the checker, never the product)."""
