/* Empty stand-in: the oracle build never writes PNG previews. */
