{
  "targets": [
    {
      "target_name": "thunderstep",
      "sources": ["thunderstep_napi.c"],
      "include_dirs": ["../../include"],
      "libraries": ["-L<(module_root_dir)/..", "-lthunderstep", "-Wl,-rpath,<(module_root_dir)/.."],
      "cflags": ["-std=c11", "-Wall"]
    }
  ]
}
