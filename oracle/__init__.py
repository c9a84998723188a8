"""ORACLE -- test infrastructure only: the FP64 CPU restatement used as the parity checker
and the timed CPU baseline.  Never imported by the product package."""
