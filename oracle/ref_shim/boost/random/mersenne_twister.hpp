// empty stand-in: the reference includes this Boost header but uses it only in commented-out code
