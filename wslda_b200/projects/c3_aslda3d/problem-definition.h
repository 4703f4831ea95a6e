/*
 * 3D TD-ASLDA with a seeded external pairing field Delta_ext(r) (NXYZ complex numbers passed
 * as extra_data: 0.2*(1 + 0.01*N(0,1)), phase 0).  No external potential.
 */
extern "C" void process_params(double *params, double *kF, double *mu, size_t extra_data_size, void *extra_data)
{
}

__device__ double v_ext(int ix, int iy, int iz, int it, int spin, double *params, size_t extra_data_size, void *extra_data)
{
    return 0.0;
}

__device__ Complex delta_ext(int ix, int iy, int iz, int it, Complex delta, double *params, size_t extra_data_size, void *extra_data)
{
    if(extra_data_size < (size_t)(2*NXYZ*sizeof(double))) return Complex(0.0, 0.0);
    const double *d = (const double *)extra_data;
    size_t i = ((size_t)ix*NY + iy)*NZ + iz;
    return Complex(d[2*i], d[2*i+1]);
}

__device__ double velocity_ext(int ix, int iy, int iz, int it, int spin, int coordinate, double *params, size_t extra_data_size, void *extra_data)
{
    return 0.0;
}

extern "C" size_t get_extra_data_size(double *params) { return (size_t)(2*NXYZ*sizeof(double)); }
extern "C" int load_extra_data(size_t extra_data_size, void *extra_data, double *params) { return 0; }

__device__ double scattering_length(int ix, int iy, int iz, int it, double *params, size_t extra_data_size, void *extra_data)
{
    return dc_sclgth;
}
