/*
 * The time-dependent Gaussian stirrer of the reference's td-gauss test family
 * (problem-definition.h of testsuite/td-gauss-bdg, -slda, -aslda, -sldae, -sldae-a1), shared by
 * the gauss_ projects:
 *
 *   V_ext(r, t) = -A s(t) exp(w_x x^2 + w_y y^2 + w_z z^2),  sign flipped for spin b when
 *   params[7] > 0.5,
 *
 * with s(t) the smooth step that rises over [t_start, t_start + T] and falls over
 * [t_stop - T, t_stop] as (1 + tanh(tan(pi/2 (2 t'/T - 1))))/2.  process_params turns the input
 * values (A in eF, widths sigma in 1/kF, times in 1/eF) into A, w = -1/(2 sigma^2) (0 for a
 * width <= 0.1) and absolute times, as pca.c:903 calls it before the constants are uploaded.
 * No pairing field, no velocity field; the scattering length is the input's sclgth.
 */
__device__ __host__ inline double gauss_ramp(double t, double T)
{
    return 0.5 * (1.0 + tanh(tan(M_PI_2 * (2.0 * t / T - 1.0))));
}

__device__ __host__ inline double gauss_window(double t, double t0, double t1, double T)
{
    if (t <= t0 || t >= t1) return 0.0;
    if (t >= t0 + T && t <= t1 - T) return 1.0;
    if (t > t0 && t < t0 + T) return gauss_ramp(t - t0, T);
    return 1.0 - gauss_ramp(t - t1 + T, T);
}

__device__ double v_ext(int ix, int iy, int iz, int it, int spin, double *params, size_t extra_data_size, void *extra_data)
{
    double x = DX * (ix - NX / 2);
    double y = DY * (iy - NY / 2);
    double z = DZ * (iz - NZ / 2);
    double t = dc_t0 + dc_dt * it;
    double s = gauss_window(t, params[4], params[5], params[6]);
    double v = -1.0 * params[0] * s * exp(params[1] * (x * x) + params[2] * (y * y) + params[3] * (z * z));
    if (spin == SPINB && params[7] > 0.5) v *= -1.0;
    return v;
}

__device__ Complex delta_ext(int ix, int iy, int iz, int it, Complex delta, double *params, size_t extra_data_size, void *extra_data)
{
    return Complex(0.0, 0.0);
}

__device__ double velocity_ext(int ix, int iy, int iz, int it, int spin, int coordinate, double *params, size_t extra_data_size, void *extra_data)
{
    return 0.0;
}

extern "C" void process_params(double *params, double *kF, double *mu, size_t extra_data_size, void *extra_data)
{
    double eF = 0.5 * kF[0] * kF[0];
    params[0] *= eF;
    for (int i = 1; i <= 3; i++) {
        double w = params[i] / kF[0];
        params[i] = (w > 0.1) ? -0.5 / (w * w) : 0.0;
    }
    params[4] /= eF;
    params[5] /= eF;
    params[6] /= eF;
}

extern "C" size_t get_extra_data_size(double *params) { return 0; }
extern "C" int load_extra_data(size_t extra_data_size, void *extra_data, double *params) { return 0; }

__device__ double scattering_length(int ix, int iy, int iz, int it, double *params, size_t extra_data_size, void *extra_data)
{
    return dc_sclgth;
}
