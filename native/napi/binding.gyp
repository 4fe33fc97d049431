{
  "targets": [
    {
      "target_name": "mutracer_b200",
      "sources": ["mutracer_b200_napi.c"],
      "include_dirs": ["../../include"],
      "libraries": ["-L<(module_root_dir)/../../mutracer_b200/_lib", "-lmutracer_b200",
                    "-Wl,-rpath,<(module_root_dir)/../../mutracer_b200/_lib"],
      "cflags": ["-std=c11", "-Wall"]
    }
  ]
}
