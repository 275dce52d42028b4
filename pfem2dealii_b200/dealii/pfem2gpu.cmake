# pfem2gpu.cmake -- build the reference (andreyypopov/pfem2dealii) with its
# particle handler on one B200.
#
# In the reference's CMakeLists.txt, after `file(GLOB src_files ...)`:
#
#     include(<this repository>/pfem2dealii_b200/dealii/pfem2gpu.cmake)
#     pfem2_b200_sources(src_files)
#
# and after `add_library(pfem2dealii SHARED ${src_files})`:
#
#     pfem2_b200_link(pfem2dealii)
#
# With -DPFEM2_WITH_B200=ON, src/pfem2particlehandler.cpp is replaced by
# pfem2particlehandler_b200.cpp (the same class over libpfem2gpu.so) and the
# library links libpfem2gpu.so; every other source, header and case driver
# compiles unchanged.  PFEM2_B200_FP32=ON selects the FP32 form.
option(PFEM2_WITH_B200 "pfem2ParticleHandler on one B200 (libpfem2gpu.so)" OFF)
option(PFEM2_B200_FP32 "with PFEM2_WITH_B200: the FP32 form instead of the FP64 form" OFF)
option(PFEM2_B200_RK2 "with PFEM2_WITH_B200: midpoint (RK2) sub-steps instead of the reference's Euler" OFF)
get_filename_component(PFEM2_B200_ROOT "${CMAKE_CURRENT_LIST_DIR}/../.." ABSOLUTE)

function(pfem2_b200_sources var)
  if(PFEM2_WITH_B200)
    set(files ${${var}})
    list(FILTER files EXCLUDE REGEX ".*/src/pfem2particlehandler\\.cpp$")
    list(APPEND files "${PFEM2_B200_ROOT}/pfem2dealii_b200/dealii/pfem2particlehandler_b200.cpp")
    set(${var} ${files} PARENT_SCOPE)
  endif()
endfunction()

function(pfem2_b200_link target)
  if(PFEM2_WITH_B200)
    target_include_directories(${target} PRIVATE "${PFEM2_B200_ROOT}/include")
    target_link_libraries(${target} PUBLIC "${PFEM2_B200_ROOT}/pfem2dealii_b200/_build/libpfem2gpu.so")
    if(PFEM2_B200_FP32)
      target_compile_definitions(${target} PRIVATE PFEM2_B200_FP32)
    endif()
    if(PFEM2_B200_RK2)
      target_compile_definitions(${target} PRIVATE PFEM2_B200_RK2)
    endif()
  endif()
endfunction()
