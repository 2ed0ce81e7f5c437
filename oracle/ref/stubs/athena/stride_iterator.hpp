// harness stand-in: not used by the sources built here
