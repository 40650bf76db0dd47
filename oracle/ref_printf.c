/*
 * Test infrastructure only (oracle build).
 *
 * printf hook linked into oracle/_ref/kfun3d_hist.out.  That binary is the
 * reference built unmodified from its own sources, except that src/kernel.c is
 * compiled with -Dprintf=kf_ref_printf so the per-step report
 * (src/kernel.c:208-212) goes through this function.  The hook widens every
 * "%g" conversion to "%.17g", which makes the printed CFL, NORM, LIFT, DRAG and
 * MOMN round-trip exactly; all other text is printed unchanged.
 */
#include <stdarg.h>
#include <stdio.h>
#include <string.h>

int kf_ref_printf(const char *fmt, ...)
{
  char wide[1024];
  size_t o = 0;
  for (const char *s = fmt; *s && o + 8 < sizeof(wide); ++s) {
    if (s[0] == '%' && s[1] == 'g') {
      memcpy(wide + o, "%.17g", 5);
      o += 5;
      ++s;
    } else {
      wide[o++] = *s;
    }
  }
  wide[o] = '\0';
  va_list ap;
  va_start(ap, fmt);
  int n = vprintf(wide, ap);
  va_end(ap);
  return n;
}
