/*
 * Small-lattice parity project.  Time-dependent external potential and a smooth complex
 * external pairing field so that every hook path (v_ext, delta_ext, it -> time) is exercised:
 *   V_ext = 0.5*w^2*r^2 + A*sin(W*t)*x/LX   (w = params[0], A = params[1], W = params[2])
 *   Delta_ext = D0*(1 + i*0.5*sin(2*pi*x/LX))*cos(2*pi*y/LY)   (D0 = params[3])
 * with x = DX*(ix-NX/2), y = DY*(iy-NY/2), z = DZ*(iz-NZ/2), t = dc_t0 + dc_dt*it.
 */
extern "C" void process_params(double *params, double *kF, double *mu, size_t extra_data_size, void *extra_data)
{
}

__device__ double v_ext(int ix, int iy, int iz, int it, int spin, double *params, size_t extra_data_size, void *extra_data)
{
    double x = DX*(ix-NX/2);
    double y = DY*(iy-NY/2);
    double z = DZ*(iz-NZ/2);
    double t = dc_t0 + dc_dt*it;
    double w = params[0];
    double v = 0.5*w*w*(x*x + y*y + z*z) + params[1]*sin(params[2]*t)*x/LX;
    if(spin==SPINB) v += 0.01*params[1];
    return v;
}

__device__ Complex delta_ext(int ix, int iy, int iz, int it, Complex delta, double *params, size_t extra_data_size, void *extra_data)
{
    double x = DX*(ix-NX/2);
    double y = DY*(iy-NY/2);
    return Complex(params[3], params[3]*0.5*sin(2.0*M_PI*x/LX))*cos(2.0*M_PI*y/LY);
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
