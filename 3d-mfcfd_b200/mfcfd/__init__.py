"""mfcfd: B200 implementation of the q-LSKUM implicit iteration."""
