// Undoes what one of the reference's OpenCL programs defined (its include
// guards and macros: real_type.h, helper.h, eos_table.h, kernel_ideal.cl,
// kernel_visc.cl, kernel_IS.cl) before the next program is included into
// the same translation unit. No include guard: included once per program.
#undef __REAL_TYPE__
#undef __HELPERH__
#undef __EOS_H__
#undef acu
#undef hbarc
#undef hbarc1
#undef hbarc3
#undef dof
#undef coef
#undef THETA
#undef IDX_PI
#undef idx
#undef idn
#undef ALONG_X
#undef ALONG_Y
#undef ALONG_Z
