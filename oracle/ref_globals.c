/* Test infrastructure: definitions of the globals that the reference mapper keeps in its
 * main.c (main.c:12-13, main.c:37-39), so that its other translation units can be linked
 * into a shared object and their functions called one by one from known-answer tests.
 * Nothing here is reference code. */
char **cmd_line = 0;
int    cmd_line_len = 0;
int    allowed_indels = 3;
int    simd_allowed_diags = 3;
int    delta_m = 9;
