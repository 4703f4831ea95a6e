/*
 * Small-lattice parity project for the external velocity field (ENABLE_VELOCITY_EXT): a
 * rotating-frame flow v = Om(t) * (-y, x) * exp(-r^2 / (2 w^2)) for both spins, with
 * Om(t) = params[6] * (1 + 0.3 sin(params[8] t)) and w = params[7], plus the time-dependent
 * trap, complex Delta_ext and x-kick of t2d_slda (params[0..3]).
 * x = DX*(ix-NX/2), y = DY*(iy-NY/2), t = dc_t0 + dc_dt*it.
 */
extern "C" void process_params(double *params, double *kF, double *mu, size_t extra_data_size, void *extra_data)
{
}

__device__ double v_ext(int ix, int iy, int iz, int it, int spin, double *params, size_t extra_data_size, void *extra_data)
{
    double x = DX*(ix-NX/2);
    double y = DY*(iy-NY/2);
    double t = dc_t0 + dc_dt*it;
    double w = params[0];
    double v = 0.5*w*w*(x*x + y*y) + params[1]*sin(params[2]*t)*x/LX;
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
    double x = DX*(ix-NX/2);
    double y = DY*(iy-NY/2);
    double t = dc_t0 + dc_dt*it;
    double om = params[6]*(1.0 + 0.3*sin(params[8]*t));
    double env = exp(-(x*x + y*y)/(2.0*params[7]*params[7]));
    if(spin==SPINB) om *= 0.8;
    if(coordinate==XAXIS) return -om*y*env;
    if(coordinate==YAXIS) return  om*x*env;
    return 0.0;
}

extern "C" size_t get_extra_data_size(double *params) { return 0; }
extern "C" int load_extra_data(size_t extra_data_size, void *extra_data, double *params) { return 0; }

__device__ double scattering_length(int ix, int iy, int iz, int it, double *params, size_t extra_data_size, void *extra_data)
{
    return dc_sclgth;
}
