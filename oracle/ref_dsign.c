/* Test infrastructure for the reference build (oracle/ref.mk).
 * The f2c translations advect.win32.c / sadvect.win32.c shipped with ParFlow
 * call libf2c's d_sign(a, b) = |a| with the sign of b, which this image does
 * not provide.  They are only reached by the IMPES solver, never by Richards. */
double d_sign(double *a, double *b)
{
  double x = (*a >= 0.0) ? *a : -*a;
  return (*b >= 0.0) ? x : -x;
}
