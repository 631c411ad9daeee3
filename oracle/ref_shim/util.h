/* Empty stand-in for a BOINC header included by the reference application; it declares nothing the oracle build uses. */
