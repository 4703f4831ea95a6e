/*
 * 2D TD-BdG with a moving Gaussian stirrer
 *   V(r,t) = A*exp(-|r-r0(t)|^2/(2*w_eff^2)),  w_eff = params[17]*w,
 *   x0(t) = R*sum_{h=1..3} [params[2h-2]*cos(h*W*t) + params[2h-1]*sin(h*W*t)]
 *   y0(t) = R*sum_{h=1..3} [params[4+2h]*cos(h*W*t) + params[5+2h]*sin(h*W*t)]
 * with A = params[12], w = params[13] (14 stirrer parameters), g = params[14],
 * R = params[15], W = params[16]; t = dc_t0 + dc_dt*it.
 */
extern "C" void process_params(double *params, double *kF, double *mu, size_t extra_data_size, void *extra_data)
{
}

__device__ __host__ inline void c4_stirrer_center(double t, const double *p, double *x0, double *y0)
{
    double sx = 0.0, sy = 0.0;
    for(int h=1; h<=3; h++)
    {
        double c = cos(h*p[16]*t), s = sin(h*p[16]*t);
        sx += p[2*h-2]*c + p[2*h-1]*s;
        sy += p[4+2*h]*c + p[5+2*h]*s;
    }
    *x0 = p[15]*sx;
    *y0 = p[15]*sy;
}

__device__ double v_ext(int ix, int iy, int iz, int it, int spin, double *params, size_t extra_data_size, void *extra_data)
{
    double x = DX*(ix-NX/2);
    double y = DY*(iy-NY/2);
    double t = dc_t0 + dc_dt*it;
    double x0, y0;
    c4_stirrer_center(t, params, &x0, &y0);
    double w = params[17]*params[13];
    double r2 = (x-x0)*(x-x0) + (y-y0)*(y-y0);
    return params[12]*exp(-r2/(2.0*w*w));
}

__device__ Complex delta_ext(int ix, int iy, int iz, int it, Complex delta, double *params, size_t extra_data_size, void *extra_data)
{
    return Complex(0.0, 0.0);
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

#include "tdwslda_functionals_framework_enable.h"
__global__ void tdwslda_compute_potentials(int it, wslda_density h_densities, wslda_potential h_potentials, double cccoeff)
{
    size_t ixyz = threadIdx.x + blockIdx.x * blockDim.x;
    int ix, iy, iz, i;
    if(ixyz<NUMBER_ELEMENT)
    {
        decode_ixyz2ixiyiz(ixyz,ix,iy,iz,i);
        double g = params[14];
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
