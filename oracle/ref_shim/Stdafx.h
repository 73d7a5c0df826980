// empty stand-in for the MSVC precompiled header of the reference project
