/*
 * 1D TD-BdG with a contact coupling g = params[0] (g = -0.5): Delta = -g*nu.
 * V_ext(x) = 0.5*omega^2*x^2 with omega = params[1] (0.05), x = DX*(ix-NX/2).
 * Delta_ext(x) is a seeded complex field handed over as extra_data (NX complex numbers).
 */
extern "C" void process_params(double *params, double *kF, double *mu, size_t extra_data_size, void *extra_data)
{
}

__device__ double v_ext(int ix, int iy, int iz, int it, int spin, double *params, size_t extra_data_size, void *extra_data)
{
    double x = DX*(ix-NX/2);
    double w = params[1];
    return 0.5*w*w*x*x;
}

__device__ Complex delta_ext(int ix, int iy, int iz, int it, Complex delta, double *params, size_t extra_data_size, void *extra_data)
{
    if(extra_data_size < (size_t)(2*NX*sizeof(double))) return Complex(0.0, 0.0);
    const double *d = (const double *)extra_data;
    return Complex(d[2*ix], d[2*ix+1]);
}

__device__ double velocity_ext(int ix, int iy, int iz, int it, int spin, int coordinate, double *params, size_t extra_data_size, void *extra_data)
{
    return 0.0;
}

extern "C" size_t get_extra_data_size(double *params) { return (size_t)(2*NX*sizeof(double)); }
extern "C" int load_extra_data(size_t extra_data_size, void *extra_data, double *params) { return 0; }

__device__ double scattering_length(int ix, int iy, int iz, int it, double *params, size_t extra_data_size, void *extra_data)
{
    return dc_sclgth;
}

#include "tdwslda_functionals_framework_enable.h"
__global__ void tdwslda_compute_potentials(int it, wslda_density h_densities, wslda_potential h_potentials, double cccoeff)
{
    size_t ixyz = threadIdx.x + blockIdx.x * blockDim.x;
    int ix, iy, iz, i;
    if(ixyz<NUMBER_ELEMENT)
    {
        decode_ixyz2ixiyiz(ixyz,ix,iy,iz,i);
        double g = params[0];
        h_potentials.V_a[ixyz] = v_ext(ix,iy,iz,it,SPINA,params,extra_data_size,extra_data);
        h_potentials.V_b[ixyz] = v_ext(ix,iy,iz,it,SPINB,params,extra_data_size,extra_data);
        h_potentials.delta[ixyz] = h_densities.nu[ixyz]*(-g);
        h_potentials.alpha_a[ixyz] = 1.0;
        h_potentials.alpha_b[ixyz] = 1.0;
    }
}

__global__ void tdwslda_compute_energy(int it, wslda_density h_densities, wslda_potential h_potentials,
                                       double *E_kin, double *E_pot, double *E_pair, double *E_curr)
{
    size_t ixyz = threadIdx.x + blockIdx.x * blockDim.x;
    if(ixyz<NUMBER_ELEMENT)
    {
        E_kin[ixyz] = 0.5*(h_potentials.alpha_a[ixyz]*h_densities.tau_a[ixyz] + h_potentials.alpha_b[ixyz]*h_densities.tau_b[ixyz])*VOLUME_ELEMENT;
        E_pot[ixyz] = 0.0;
        E_pair[ixyz] = (h_potentials.delta[ixyz]*thrust::conj(h_densities.nu[ixyz])).real()*(-0.5)*VOLUME_ELEMENT;
        E_curr[ixyz] = 0.0;
    }
}
#include "tdwslda_functionals_framework_disable.h"
