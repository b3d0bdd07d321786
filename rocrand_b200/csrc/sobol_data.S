/* Embeds rocrand_b200/data/sobol_params.bin (Joe-Kuo Sobol parameters, see
   make_sobol_params.py) into librocrand.so. */
    .section .note.GNU-stack,"",@progbits
    .section .rodata
    .globl rb200_sobol_params_begin
    .globl rb200_sobol_params_end
    .hidden rb200_sobol_params_begin
    .hidden rb200_sobol_params_end
    .p2align 4
rb200_sobol_params_begin:
    .incbin "sobol_params.bin"
rb200_sobol_params_end:
