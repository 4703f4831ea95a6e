/*
 * 3D TD-SLDA vortex: Delta_ext = D0*tanh(rho/xi)*exp(i*phi) (D0 = params[0] = 0.2,
 * xi = params[1] = 5), rho = distance from the z axis through the lattice centre.
 * Stirrer: a Gaussian beam along z, V = A*exp(-|r_perp - c(t)|^2/(2 w^2)), A = params[2] = 0.3,
 * w = params[3] = 3, circling at radius params[4] = 10 with angular velocity params[5] = 0.2.
 */
extern "C" void process_params(double *params, double *kF, double *mu, size_t extra_data_size, void *extra_data)
{
}

__device__ double v_ext(int ix, int iy, int iz, int it, int spin, double *params, size_t extra_data_size, void *extra_data)
{
    double x = DX*(ix-NX/2);
    double y = DY*(iy-NY/2);
    double t = dc_t0 + dc_dt*it;
    double x0 = params[4]*cos(params[5]*t);
    double y0 = params[4]*sin(params[5]*t);
    double r2 = (x-x0)*(x-x0) + (y-y0)*(y-y0);
    return params[2]*exp(-r2/(2.0*params[3]*params[3]));
}

__device__ Complex delta_ext(int ix, int iy, int iz, int it, Complex delta, double *params, size_t extra_data_size, void *extra_data)
{
    double x = DX*(ix-NX/2);
    double y = DY*(iy-NY/2);
    double r = sqrt(x*x + y*y);
    if(r == 0.0) return Complex(0.0, 0.0);
    double a = params[0]*tanh(r/params[1]);
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
