/* Embeds rocrand_b200/data/sobol_params.bin (the Joe-Kuo Sobol parameters) into liborc.so
   (test infrastructure only). */
    .section .note.GNU-stack,"",@progbits
    .section .rodata
    .globl orc_sobol_params_begin
    .p2align 4
orc_sobol_params_begin:
    .incbin "sobol_params.bin"
