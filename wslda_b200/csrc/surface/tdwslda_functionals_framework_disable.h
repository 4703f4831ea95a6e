/* Closes the block opened by tdwslda_functionals_framework_enable.h
 * (hpc-engine/tdwslda_functionals_framework_disable.h). */
#undef params
#undef extra_data
#undef extra_data_size
#undef NUMBER_ELEMENT
#undef VOLUME_ELEMENT
#undef decode_ixyz2ixiyiz
