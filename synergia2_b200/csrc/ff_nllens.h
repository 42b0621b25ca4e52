// Thin nonlinear lens (Danilov-Nagaitsev elliptic potential): nllens_unit
// ff_algorithm.h:1180-1270, shared by the host (design particle) and the
// particle kernels.  k = {1/cnll, -knll/cnll}; with z = (x + i y)/cnll the
// kick is k[1] (Re, -Im) of z/(1 - z^2) + asin(z)/(1 - z^2), where the square
// root of 1 - z^2 is taken with a non-negative imaginary part and
// asin(z) = -i log(i z + sqrt(1 - z^2)) -- the arithmetic the reference
// runs.  On the cut (y = 0, |x| >= cnll) the angles become NaN.
//
// Included inside a namespace; the includer defines SB2_FF.
#ifndef SB2_FF
#error "define SB2_FF before including ff_nllens.h"
#endif

SB2_FF void nllens_unit(double x, double& xp, double y, double& yp, const double* k)
{
    const double icnll = k[0], kick = k[1];
    const double zr = x * icnll, zi = y * icnll;
    if (zi == 0 && (zr >= 1.0 || zr <= -1.0)) {
        xp = __builtin_nan("");
        yp = __builtin_nan("");
        return;
    }
    const double cr = 1.0 - zr * zr + zi * zi;
    const double ci = -2.0 * zr * zi;
    const double croot_r = sqrt(0.5 * (cr + sqrt(cr * cr + ci * ci)));
    const double croot_i = sqrt(0.5 * (-cr + sqrt(cr * cr + ci * ci)));
    const double co_r = croot_r - zi;
    const double co_i = croot_i + zr;
    const double r = sqrt(co_r * co_r + co_i * co_i);
    const double theta = (co_r > 0) ? atan(co_i / co_r) + 0.0 : atan(co_i / co_r) + 3.14159265358979323846;
    const double as_r = theta;   // -i log(co)
    const double as_i = -log(r);
    const double c2r = croot_r * croot_r - croot_i * croot_i;
    const double c2i = 2.0 * croot_r * croot_i;
    const double d1r = (c2r * zr + c2i * zi) / (c2r * c2r + c2i * c2i);
    const double d1i = (c2r * zi - c2i * zr) / (c2r * c2r + c2i * c2i);
    const double d2r = (c2r * as_r + c2i * as_i) / (c2r * c2r + c2i * c2i);
    const double d2i = (c2r * as_i - c2i * as_r) / (c2r * c2r + c2i * c2i);
    xp = xp + kick * (d1r + d2r);
    yp = yp + -kick * (d1i + d2i);
}
