/*
 * Small-lattice parity project for the external velocity field in BdG mode: a flow along x,
 * v_a = params[6]*sin(2 pi x/LX + params[7] t), v_b = 0.5 * v_a, with the time-dependent trap
 * and complex Delta_ext of the other parity projects (params[0..3]).
 * x = DX*(ix-NX/2), t = dc_t0 + dc_dt*it.
 */
extern "C" void process_params(double *params, double *kF, double *mu, size_t extra_data_size, void *extra_data)
{
}

__device__ double v_ext(int ix, int iy, int iz, int it, int spin, double *params, size_t extra_data_size, void *extra_data)
{
    double x = DX*(ix-NX/2);
    double t = dc_t0 + dc_dt*it;
    double w = params[0];
    double v = 0.5*w*w*x*x + params[1]*sin(params[2]*t)*x/LX;
    if(spin==SPINB) v += 0.01*params[1];
    return v;
}

__device__ Complex delta_ext(int ix, int iy, int iz, int it, Complex delta, double *params, size_t extra_data_size, void *extra_data)
{
    double x = DX*(ix-NX/2);
    return Complex(params[3], params[3]*0.5*sin(2.0*M_PI*x/LX));
}

__device__ double velocity_ext(int ix, int iy, int iz, int it, int spin, int coordinate, double *params, size_t extra_data_size, void *extra_data)
{
    double x = DX*(ix-NX/2);
    double t = dc_t0 + dc_dt*it;
    if(coordinate!=XAXIS) return 0.0;
    double v = params[6]*sin(2.0*M_PI*x/LX + params[7]*t);
    return (spin==SPINB) ? 0.5*v : v;
}

extern "C" size_t get_extra_data_size(double *params) { return 0; }
extern "C" int load_extra_data(size_t extra_data_size, void *extra_data, double *params) { return 0; }

__device__ double scattering_length(int ix, int iy, int iz, int it, double *params, size_t extra_data_size, void *extra_data)
{
    return dc_sclgth;
}
