# Test infrastructure: writes the reference's db/db_impl.cc with its
# DoCompactionWork definitions replaced by an include of the drop-in body.
#
#   awk -v INC=<path of luda_b200/host/do_compaction_work.cc> -f patch_db_impl.awk db_impl.cc
#
# db/db_impl.cc:1059-1592 reads
#   #if !(GPU_ACCELERATE)
#   Status DBImpl::DoCompactionWork(CompactionState* compact) { ...CPU... }
#   #else
#   ...GPU...
#   #endif
# The CPU body (nested #if/#endif included) is dropped and the #if becomes
# `#if 1` around the include, so the GPU body under #else is never compiled.
# Everything else is copied unchanged; GPU_ACCELERATE is set to 0 by sed
# beforehand, so WriteLevel0Table keeps the reference's BuildTable.
state == 0 && /^#if !\(GPU_ACCELERATE\)$/ {
  if ((getline nxt) > 0) {
    if (nxt ~ /^Status DBImpl::DoCompactionWork\(CompactionState\* compact\) \{$/) {
      print "#if 1  // DoCompactionWork: the luda_b200 drop-in"
      print "#include \"" INC "\""
      state = 1
      depth = 0
      next
    }
    print
    print nxt
    next
  }
}
state == 1 {
  if ($0 ~ /^#if/) depth++
  else if ($0 ~ /^#endif/) depth--
  else if ($0 ~ /^#else$/ && depth == 0) { print; state = 2 }
  next
}
{ print }
END { if (state != 2) { print "patch_db_impl.awk: DoCompactionWork not found" > "/dev/stderr"; exit 1 } }
