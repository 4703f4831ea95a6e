/*
 * 2D TD-SLDA: harmonic trap V = 0.5*omega^2*r^2 (omega = params[0] = 0.04) and an imprinted
 * vortex Delta_ext = D0*tanh(r/xi)*exp(i*phi) (D0 = params[1] = 0.25, xi = params[2] = 4),
 * centred at the lattice centre; x = DX*(ix-NX/2), y = DY*(iy-NY/2).
 */
extern "C" void process_params(double *params, double *kF, double *mu, size_t extra_data_size, void *extra_data)
{
}

__device__ double v_ext(int ix, int iy, int iz, int it, int spin, double *params, size_t extra_data_size, void *extra_data)
{
    double x = DX*(ix-NX/2);
    double y = DY*(iy-NY/2);
    double w = params[0];
    return 0.5*w*w*(x*x + y*y);
}

__device__ Complex delta_ext(int ix, int iy, int iz, int it, Complex delta, double *params, size_t extra_data_size, void *extra_data)
{
    double x = DX*(ix-NX/2);
    double y = DY*(iy-NY/2);
    double r = sqrt(x*x + y*y);
    double a = params[1]*tanh(r/params[2]);
    if(r == 0.0) return Complex(0.0, 0.0);
    return Complex(a*x/r, a*y/r);
}

__device__ double velocity_ext(int ix, int iy, int iz, int it, int spin, int coordinate, double *params, size_t extra_data_size, void *extra_data)
{
    return 0.0;
}

extern "C" size_t get_extra_data_size(double *params) { return 0; }
extern "C" int load_extra_data(size_t extra_data_size, void *extra_data, double *params) { return 0; }

__device__ double scattering_length(int ix, int iy, int iz, int it, double *params, size_t extra_data_size, void *extra_data)
{
    return dc_sclgth;
}
