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

/* CUSTOMEDF: contact BdG coupling g = params[4] plus a density-dependent mean field
 * U_s = params[5]*rho_s (spin-diagonal Hartree-like term). */
#include "tdwslda_functionals_framework_enable.h"
__global__ void tdwslda_compute_potentials(int it, wslda_density h_densities, wslda_potential h_potentials, double cccoeff)
{
    size_t ixyz = threadIdx.x + blockIdx.x * blockDim.x;
    int ix, iy, iz, i;
    if(ixyz<NUMBER_ELEMENT)
    {
        decode_ixyz2ixiyiz(ixyz,ix,iy,iz,i);
        double g = params[4];
        h_potentials.V_a[ixyz] = v_ext(ix,iy,iz,it,SPINA,params,extra_data_size,extra_data) + params[5]*h_densities.rho_b[ixyz];
        h_potentials.V_b[ixyz] = v_ext(ix,iy,iz,it,SPINB,params,extra_data_size,extra_data) + params[5]*h_densities.rho_a[ixyz];
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
        E_pot[ixyz] = params[5]*h_densities.rho_a[ixyz]*h_densities.rho_b[ixyz]*VOLUME_ELEMENT;
        E_pair[ixyz] = (h_potentials.delta[ixyz]*thrust::conj(h_densities.nu[ixyz])).real()*(-0.5)*VOLUME_ELEMENT;
        E_curr[ixyz] = 0.0;
    }
}
#include "tdwslda_functionals_framework_disable.h"
