// Process-wide count of the library's kernel launches (bemgpu_kernel_launches):
// every launch site adds what it launched; a captured graph adds its kernel
// count per replay.
#pragma once
#ifdef __cplusplus
extern "C" {
#endif
void bem_count_launches(unsigned long long n);
#ifdef __cplusplus
}
#endif
