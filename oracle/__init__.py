"""ORACLE package -- test infrastructure only (the checker).  Never imported by the product."""
