"""ctpwa_b200 package (API is added below)."""
