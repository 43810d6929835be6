/* empty stand-in: the compiled STIR file needs no Boost configuration */
