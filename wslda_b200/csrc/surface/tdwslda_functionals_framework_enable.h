/*
 * User-surface helper: names that hook code in a project's problem-definition.h uses inside
 * device functions (params, extra_data, NUMBER_ELEMENT, VOLUME_ELEMENT, decode_ixyz2ixiyiz).
 * Same macro names and meaning as hpc-engine/tdwslda_functionals_framework_enable.h:1-41, so an
 * unmodified user file compiles against this library.  Paired with ..._disable.h.
 */
#define params dc_params
#define extra_data dc_extra_data
#define extra_data_size dc_extra_data_size

#if CODEDIM==1
#define NUMBER_ELEMENT NX
#define VOLUME_ELEMENT (DXYZ*NY*NZ)
#elif CODEDIM==2
#define NUMBER_ELEMENT NXY
#define VOLUME_ELEMENT (DXYZ*NZ)
#elif CODEDIM==3
#define NUMBER_ELEMENT NXYZ
#define VOLUME_ELEMENT (DXYZ)
#else
#error CODEDIM NOT SPECIFIED
#endif

#if CODEDIM==3
#define decode_ixyz2ixiyiz(ixyz,_ix,_iy,_iz,i) ixyz2ixiyiz(ixyz,_ix,_iy,_iz,i)
#elif CODEDIM==2
#define decode_ixyz2ixiyiz(ixyz,_ix,_iy,_iz,i) ixy2ixiy2d(ixyz,_ix,_iy) _iz=0;
#else
#define decode_ixyz2ixiyiz(ixyz,_ix,_iy,_iz,i) _ix=(int)(ixyz); _iy=0; _iz=0;
#endif
