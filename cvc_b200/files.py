"""Propagator file naming of the reference (get_filename, cvc_utils.c:
2143-2198), for callers that feed the contraction from CVC's file sets.

The 60 "up" columns of one source are files  <prefix>.<Nconf>.<nu>.<sc>.inverted
(format 0): nu = 0..3 is the source shifted by +mu, nu = 4 the unshifted
source (cvc_exact2_xspace.c:401-430 reads them as fields[12*nu + sc]).
"""


def get_filename(nu, sc, sign, *, filename_prefix, filename_prefix2, Nconf, format,
                 source_location, T_global, LX_global, LY_global, LZ_global):
    """Same string as the reference for formats 0, 2, 3, 4 (format 1 and
    unknown formats produce no name there; here they raise)."""
    sx = [source_location // (LX_global * LY_global * LZ_global),
          (source_location % (LX_global * LY_global * LZ_global)) // (LY_global * LZ_global),
          (source_location % (LY_global * LZ_global)) // LZ_global,
          source_location % LZ_global]
    L = [T_global, LX_global, LY_global, LZ_global]

    def shifted():
        s = list(sx)
        if nu != 4:
            s[nu] = (s[nu] + 1) % L[nu]
        return s

    if format == 0:
        if sign == 1:
            return "%s.%.4d.%.2d.%.2d.inverted" % (filename_prefix, Nconf, nu, sc)
        if sign == -1:
            return "%s.%.4d.%.2d.%.2d.inverted" % (filename_prefix2, Nconf, nu, sc)
        if sign == 0:
            s = shifted()
            return "%s.%.4d.t%.2dx%.2dy%.2dz%.2d.%.2d.inverted" % (
                filename_prefix, Nconf, s[0], s[1], s[2], s[3], sc)
    elif format == 2:
        s = shifted()
        mass = "pmass" if sign == 1 else "nmass"
        return "%s.%.4d.t%.2dx%.2dy%.2dz%.2ds%.2dc%.2d.%s.%s.inverted" % (
            filename_prefix, Nconf, s[0], s[1], s[2], s[3], sc // 3, sc % 3, mass,
            filename_prefix2)
    elif format == 3:
        s = shifted()
        mass = "pmass" if sign == 1 else "nmass"
        return "%s.%.4d.t%.2dx%.2dy%.2dz%.2d.%s.%s.%.2d.inverted" % (
            filename_prefix, Nconf, s[0], s[1], s[2], s[3], mass, filename_prefix2, sc)
    elif format == 4:
        return "%s.%.4d.%.2d.inverted" % (filename_prefix if sign == 1 else filename_prefix2,
                                          Nconf, sc)
    raise ValueError(f"no file name for format {format}, sign {sign}")
