/* Stand-in for the Cactus arguments header (empty). */
