/* Embeds the XORWOW subsequence jump polynomials (derived at build time by
   rocrand_b200/data/make_xorwow_jump.c) into librocrand.so. */
    .section .note.GNU-stack,"",@progbits
    .section .rodata
    .globl rb200_xorwow_jump_begin
    .globl rb200_xorwow_jump_end
    .hidden rb200_xorwow_jump_begin
    .hidden rb200_xorwow_jump_end
    .p2align 4
rb200_xorwow_jump_begin:
    .incbin "xorwow_jump.bin"
rb200_xorwow_jump_end:
