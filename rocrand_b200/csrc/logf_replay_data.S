/* Embeds logf_replay.bin (the host-logf replay table of the inverse-erf normal, written at
   build time by rocrand_b200/data/make_logf_replay.cpp) into librocrand.so. */
    .section .note.GNU-stack,"",@progbits
    .section .rodata
    .globl rb200_logf_replay_begin
    .globl rb200_logf_replay_end
    .hidden rb200_logf_replay_begin
    .hidden rb200_logf_replay_end
    .p2align 4
rb200_logf_replay_begin:
    .incbin "logf_replay.bin"
rb200_logf_replay_end:
